"""Build recipe for the checker libraries (TEST INFRASTRUCTURE).

* ``oracle/liboracle.so``  - the plain-C restatement (ga_oracle.c), built from this repository alone, so it also
  builds on a machine without the reference sources.
* ``oracle/_ref/libga_ref.so`` - the reference's own CPU code (src/graph.h, src/densest.h, src/dsg.h of
  VijayPraneethSai/graph_analyzer) compiled where it lies, through the wrappers in ref_shim.cpp. Built only when the
  reference tree is present; the output is git-ignored and travels with the working tree.

Usage: ``python oracle/build_oracle.py [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# root of the reference's source tree (read only); GA_REFERENCE_ROOT overrides the default location
REF_ROOT = os.environ.get("GA_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libga_ref.so")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "ga_oracle.c")
    hdr = os.path.join(HERE, "ga_oracle.h")
    if force or _stale(ORACLE_SO, [src, hdr, __file__]):
        cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", src, "-o", ORACLE_SO]
        subprocess.check_call(cmd)
    return ORACLE_SO


def build_ref(force: bool = False) -> str | None:
    """Compiles the reference's headers through ref_shim.cpp. Returns None when the reference tree is absent."""
    if not os.path.isdir(REF_SRC):
        return REF_SO if os.path.exists(REF_SO) else None
    shim = os.path.join(HERE, "ref_shim.cpp")
    deps = [shim, __file__] + [os.path.join(REF_SRC, h) for h in ("graph.h", "densest.h", "dsg.h")]
    if force or _stale(REF_SO, deps):
        os.makedirs(os.path.dirname(REF_SO), exist_ok=True)
        cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-I", REF_SRC, shim, "-o", REF_SO]
        subprocess.check_call(cmd)
    return REF_SO


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_ref(force))
