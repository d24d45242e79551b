"""Builds libga_b200.so in-tree (graph_analyzer_b200/_lib/) for sm_100a with nvcc, and the command-line drivers.

Every .cu / .cpp under csrc/ is compiled to an object in _build/ (in parallel), then linked into one shared library
with the CUDA runtime linked statically, so the library does not depend on which libcudart a host process (e.g. torch)
has loaded. The drivers under cli/ (ga_tc, ga_densest, ga_dsg) are plain C++ over the C ABI, linked against the
library into graph_analyzer_b200/_bin/. Usage: ``python -m graph_analyzer_b200.build [--force] [--verbose-ptxas]``.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
BIN_DIR = os.path.join(PKG, "_bin")
CLI_DIR = os.path.join(PKG, "cli")
CLIS = ["ga_tc", "ga_densest", "ga_dsg"]
BUILD_DIR = os.path.join(ROOT, "_build")
LIB = os.path.join(OUT_DIR, "libga_b200.so")
# the generators alone (no CUDA): for processes that must not load libga_b200 (bench.py's reference arm)
GEN_LIB = os.path.join(OUT_DIR, "libga_gen.so")
GEN_SOURCES = [os.path.join(CSRC, "ga_gen.cpp"), os.path.join(CSRC, "standalone", "ga_gen_errors.cpp")]
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
    deps = [src, __file__] + _headers()
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [_nvcc(), "-c", src, "-o", obj, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-I", INCLUDE, "-I", CSRC,
           "-Xcompiler", "-fPIC,-fopenmp,-O3", "--expt-relaxed-constexpr"]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    subprocess.check_call(cmd)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    if force:
        for o in glob.glob(os.path.join(BUILD_DIR, "*.o")):
            os.remove(o)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [_nvcc(), "-shared", *ARCH, "-o", LIB, *objs, "-cudart", "static", "-Xcompiler", "-fopenmp",
               "-lgomp"]
        subprocess.check_call(cmd)
    build_gen(force)
    build_cli(force)
    return LIB


def build_gen(force: bool = False) -> str:
    """libga_gen.so: the seeded R-MAT sampler and id permutation of ga_gen.cpp, host C++ only."""
    deps = GEN_SOURCES + [__file__, os.path.join(CSRC, "ga_internal.h"), os.path.join(INCLUDE, "graph_analyzer_b200.h")]
    if force or not os.path.exists(GEN_LIB) or any(os.path.getmtime(d) > os.path.getmtime(GEN_LIB) for d in deps):
        subprocess.check_call(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-I", INCLUDE, "-I", CSRC,
                               *GEN_SOURCES, "-o", GEN_LIB])
    return GEN_LIB


def build_cli(force: bool = False) -> list[str]:
    """Compiles the drivers (host C++ only) against the in-tree library; rpath points at ../_lib."""
    os.makedirs(BIN_DIR, exist_ok=True)
    deps = [LIB, __file__, os.path.join(CLI_DIR, "cli_common.hpp"), os.path.join(INCLUDE, "graph_analyzer_b200.h"),
            os.path.join(INCLUDE, "ga", "graph_analyzer.hpp")]
    out = []
    for name in CLIS:
        src = os.path.join(CLI_DIR, name + ".cpp")
        exe = os.path.join(BIN_DIR, name)
        out.append(exe)
        if (not force and os.path.exists(exe)
                and all(os.path.getmtime(exe) >= os.path.getmtime(d) for d in deps + [src])):
            continue
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, "-I", CLI_DIR, src, "-o", exe,
                               "-L", OUT_DIR, "-lga_b200", "-Wl,-rpath,$ORIGIN/../_lib"])
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--verbose-ptxas" in sys.argv))
