// Shared by the C-ABI translation units: the thread-local last error and the guard that turns
// every C++ exception into a status code, as ybus_ffi turns panics and errors into status codes
// with a thread-local message (ybus_ffi/src/lib.rs:44-73, ybus_ffi/src/status.rs:1-60).
#pragma once

#include <cstdint>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "host/sparse.hpp"

namespace yb {

void set_last_error(const std::string &message);
void clear_last_error();

template <class F> int32_t guard(F &&body) {
  try {
    clear_last_error();
    return body();
  } catch (const host::Error &e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("out of host memory");
    return host::kInternal;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return host::kInternal;
  } catch (...) {
    set_last_error("unknown error");
    return host::kInternal;
  }
}

inline void require(bool ok, const char *what, int status = host::kInvalidArgument) {
  if (!ok) throw host::Error(status, what);
}

}  // namespace yb
