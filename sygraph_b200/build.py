"""Build recipe for libsygraph_b200.so (sm_100a) and the C++ API test programs.

Every CUDA source is compiled by nvcc for ``sm_100a`` only and linked in-tree
into ``sygraph_b200/libsygraph_b200.so`` so the library travels with the
source tree.  Object files go to ``_build/`` (not committed).  Sources are
rebuilt only when a source or header is newer than the library.

Usage: ``python sygraph_b200/build.py [--force] [-j N]`` (run as a script: importing the
package itself needs the built library).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libsygraph_b200.so"
CPP_TESTS = ROOT / "tests" / "cpp"
CPP_TEST_BIN = CPP_TESTS / "bin"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", "/usr/bin/g++"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++20",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "--extended-lambda",
    "-Xcompiler",
    "-fPIC,-fopenmp,-O3",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]
CXX_FLAGS = ["-O3", "-std=c++20", "-fPIC", "-fopenmp", f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libsygraph_b200.so")


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.rglob("*.h*")) +
                  list(INCLUDE.rglob("*.cuh")))


def _newest(paths) -> float:
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if src.suffix == ".cu":
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["/usr/bin/g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build_library(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Compile and link libsygraph_b200.so; returns its path."""
    srcs = _sources()
    hdr_time = _newest(_headers())
    BUILD.mkdir(exist_ok=True)
    stale = []
    for s in srcs:
        obj = BUILD / (s.name + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(s.stat().st_mtime, hdr_time):
            stale.append(s)
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    if stale:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            list(ex.map(lambda s: _compile(s, verbose), stale))
    objs = [BUILD / (s.name + ".o") for s in srcs]
    if force or stale or not LIB.exists() or LIB.stat().st_mtime < _newest(objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


def build_cpp_tests(force: bool = False, jobs: int | None = None, verbose: bool = False) -> list[Path]:
    """Compile tests/cpp/*.cu (programs written against the C++ header API)."""
    srcs = sorted(CPP_TESTS.glob("*.cu"))
    if not srcs:
        return []
    CPP_TEST_BIN.mkdir(parents=True, exist_ok=True)
    hdr_time = max(_newest(_headers()), LIB.stat().st_mtime if LIB.exists() else 0.0)

    def one(src: Path) -> Path:
        exe = CPP_TEST_BIN / src.stem
        if not force and exe.exists() and exe.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
            return exe
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, str(src), "-o", str(exe), f"-L{PKG}", "-lsygraph_b200",
               f"-Xlinker", f"-rpath,{PKG}", "-Xlinker", "-rpath,$ORIGIN/../../../sygraph_b200"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
        return exe

    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        return list(ex.map(one, srcs))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--no-cpp-tests", action="store_true")
    a = ap.parse_args()
    lib = build_library(a.force, a.j, a.v)
    print(f"built {lib}")
    if not a.no_cpp_tests:
        for exe in build_cpp_tests(a.force, a.j, a.v):
            print(f"built {exe}")


if __name__ == "__main__":
    main()
