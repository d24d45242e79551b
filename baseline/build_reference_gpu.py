"""Builds the reference's own GPU drivers (gpu_tc, gpu_densest, gpu_dsg) from its sources for sm_100a, with the flags
of its Makefile (-O3 -std=c++17 -Xcompiler -fopenmp), into baseline/_ref/bin/. They are run only as a comparison
(`bench.py --workload reference-gpu`): the reference's kernels v1-v9 on the same graph and the same GPU.

Usage: python baseline/build_reference_gpu.py [reference_root]   (default: $GA_REFERENCE_ROOT, else /root/reference)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "bin")
PROGRAMS = ["gpu_tc", "gpu_densest", "gpu_dsg"]
REF_ROOT = os.environ.get("GA_REFERENCE_ROOT", "/root/reference")


def build(ref_root: str = REF_ROOT) -> list[str]:
    src = os.path.join(ref_root, "src")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"{src} not found")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(OUT, exist_ok=True)
    out = []
    for name in PROGRAMS:
        exe = os.path.join(OUT, name)
        cu = os.path.join(src, name + ".cu")
        deps = [cu] + [os.path.join(src, h) for h in os.listdir(src) if h.endswith((".h", ".cuh"))]
        if not (os.path.exists(exe) and all(os.path.getmtime(exe) >= os.path.getmtime(d) for d in deps)):
            subprocess.check_call([nvcc, "-O3", "-std=c++17", "-arch=sm_100a", "-Xcompiler", "-fopenmp", cu, "-o", exe])
        out.append(exe)
    return out


if __name__ == "__main__":
    print("\n".join(build(sys.argv[1] if len(sys.argv) > 1 else REF_ROOT)))
