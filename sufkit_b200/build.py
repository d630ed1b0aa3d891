"""Build recipe for the sufgpu shared library (sm_100a, built in-tree).

``python -m sufkit_b200.build`` compiles ``csrc/*.cu`` and ``csrc/*.cpp`` into
``sufkit_b200/libsufgpu.so`` with nvcc.  nvcc cross-compiles for sm_100a on a
machine without a GPU, so this runs anywhere the CUDA toolkit is installed.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libsufgpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    stamp = LIB.stat().st_mtime
    inputs = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp"))
    inputs += sorted((HERE.parent / "include").rglob("*.h"))
    return all(p.stat().st_mtime <= stamp for p in inputs)


DRIVER = HERE.parent / "tests" / "cpp" / "cuda_backend_driver"
DSS_LIB = HERE / "libdivsufsort_cuda.so"
DSS_SRC = HERE / "integration" / "divsufsort_cuda.cpp"


def build_divsufsort_abi(verbose: bool = False) -> Path:
    """libdivsufsort_cuda.so: divsufsort / divsufsort64 with libdivsufsort's
    exact C ABI, linked against libsufgpu.so."""
    inputs = [DSS_SRC, HERE.parent / "include" / "sufgpu" / "divsufsort_cuda.h", LIB]
    if DSS_LIB.exists() and DSS_LIB.stat().st_mtime >= max(p.stat().st_mtime for p in inputs):
        return DSS_LIB
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-fPIC", "-shared",
           "-fvisibility=hidden", f"-I{HERE.parent / 'include'}", "-o", str(DSS_LIB),
           str(DSS_SRC), f"-L{HERE}", "-lsufgpu", "-Wl,-rpath,$ORIGIN",
           "-Wl,--exclude-libs,ALL"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return DSS_LIB


def build_driver(verbose: bool = False) -> Path:
    """The C++ adapter's test driver (tests/cpp), linked against libsufgpu.so."""
    src = DRIVER.with_suffix(".cpp")
    if DRIVER.exists() and DRIVER.stat().st_mtime >= max(src.stat().st_mtime, LIB.stat().st_mtime):
        return DRIVER
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-o", str(DRIVER), str(src),
           f"-L{HERE}", "-lsufgpu", f"-Wl,-rpath,{HERE}"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        build_driver(verbose)
        build_divsufsort_abi(verbose)
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-shared", "-o", str(LIB) + ".tmp",
           *map(str, sources()), "-lz"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    build_driver(verbose)
    build_divsufsort_abi(verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
