"""Builds the package's native libraries in-tree with g++ and nvcc (sm_100a, B200):

- ``libybhost.so``: the host factor producer and the last-error store (C++, no CUDA), the only
  library a host-only caller (the CPU reference arm, the host tests) loads;
- ``libybgpu.so``: the plan and layout builders (C++), the CUDA kernels and the C ABI of the GPU
  path; it depends on ``libybhost.so`` (found beside it through its run path);
- ``libybcompare.so``: for comparison only, ybus_cuda's cuSPARSE route re-created on the same
  arrays; no solve of ``libybgpu.so`` loads it.

They are built in place (``ybus_b200/*.so``) so they travel with the source tree; nothing is
cached outside the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
HOST_LIB = HERE / "libybhost.so"
LIB = HERE / "libybgpu.so"
COMPARE_LIB = HERE / "libybcompare.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_SOURCES = ["host/factor.cpp", "host/colamd.cpp", "capi_host.cpp"]


def host_sources() -> list[Path]:
    return [CSRC / s for s in HOST_SOURCES]


def sources() -> list[Path]:
    """The sources of libybgpu.so."""
    host = set(host_sources())
    files = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    return [f for f in files if f not in host]


def compare_sources() -> list[Path]:
    return sorted((CSRC / "compare").glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.rglob("*.hpp")) + sorted(CSRC.rglob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _fresh(lib: Path, inputs: list[Path]) -> bool:
    if not lib.exists():
        return False
    built = lib.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in inputs)


def up_to_date() -> bool:
    return (_fresh(HOST_LIB, host_sources() + _headers()) and _fresh(LIB, sources() + _headers() + [HOST_LIB])
            and _fresh(COMPARE_LIB, compare_sources()))


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    if path.exists():
        return str(path)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    return found


def _compile(srcs: list[Path], objdir: Path, verbose: bool) -> list[Path]:
    common = ["-std=c++17", "-O3", "-I", str(CSRC), "-I", str(INCLUDE)]
    objs, procs = [], []
    for src in srcs:
        rel = src.relative_to(CSRC).with_suffix("")
        obj = objdir / (str(rel).replace("/", "_") + (".cu.o" if src.suffix == ".cu" else ".o"))
        if src.suffix == ".cu":
            cmd = [nvcc(), *ARCH, "-lineinfo", "--expt-relaxed-constexpr", *common, "-Xcompiler", "-fPIC", "-c",
                   str(src), "-o", str(obj)]
        else:
            cmd = ["g++", *common, "-fPIC", "-Wall", "-I", str(Path(nvcc()).parent.parent / "include"), "-c", str(src),
                   "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    failed = []
    for proc, src in procs:
        out, _ = proc.communicate()
        if proc.returncode != 0:
            failed.append(f"{src.name}:\n{out.decode(errors='replace')}")
        elif verbose and out:
            print(out.decode(errors="replace"), file=sys.stderr)
    if failed:
        raise RuntimeError("build failed:\n" + "\n".join(failed))
    return objs


def _link(cmd: list[str], target: Path) -> None:
    tmp = target.with_suffix(".so.tmp")
    res = subprocess.run([*cmd, "-o", str(tmp)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link of {target.name} failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, target)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    host_objs = _compile(host_sources(), objdir, verbose)
    _link(["g++", "-shared", "-Wl,-soname,libybhost.so", *map(str, host_objs), "-lpthread"], HOST_LIB)
    gpu_objs = _compile(sources(), objdir, verbose)
    _link([nvcc(), *ARCH, "-shared", *map(str, gpu_objs), "-L", str(HERE), "-lybhost", "-Xlinker", "-rpath=$ORIGIN",
           "-lpthread"], LIB)
    cmp_objs = _compile(compare_sources(), objdir, verbose)
    _link([nvcc(), *ARCH, "-shared", *map(str, cmp_objs), "-ldl"], COMPARE_LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
