"""Builds libybgpu.so in-tree with nvcc for sm_100a (B200).

The library holds the host factor producer (C++), the plan builder (C++) and the CUDA kernels
with their C ABI. It is built in place (``ybus_b200/libybgpu.so``) so it travels with the
source tree; nothing is cached outside the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libybgpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources() -> list[Path]:
    files = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")) + sorted((CSRC / "host").glob("*.cpp"))
    return files


def _inputs() -> list[Path]:
    return sources() + sorted(CSRC.rglob("*.hpp")) + sorted(CSRC.rglob("*.cuh")) + [HERE.parent / "include" / "ybgpu.h"]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    built = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in _inputs())


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    if path.exists():
        return str(path)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    return found


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    common = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I", str(HERE.parent / "include")]
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.stem + (".cu.o" if src.suffix == ".cu" else ".o"))
        if src.suffix == ".cu":
            cmd = [nvcc(), *ARCH, "-lineinfo", "--expt-relaxed-constexpr", *common, "-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-Wall", "-I", str(CSRC), "-I", str(HERE.parent / "include"),
                   "-I", str(Path(nvcc()).parent.parent / "include"), "-c", str(src), "-o", str(obj)]
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
    tmp = LIB.with_suffix(".so.tmp")
    link = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
