"""Regenerates the golden fixtures in this folder (run in a container that has the reference tree).

1. The reference's own fixture generators (scripts/gen_test_graph.py, scripts/gen_powerlaw.py of
   VijayPraneethSai/graph_analyzer, with the arguments of its scripts/test_emu.sh:16-19) write the four SNAP-style text
   graphs and print their brute-force triangle counts; both are kept here (``<name>.txt``, ``golden.json``).
2. The reference's own CPU code, compiled from its headers (oracle/_ref/libga_ref.so), loads each text graph with
   load_graph and produces the expected outputs: CSR, triangle count, per-edge support (for_each_triangle),
   triangle degrees, batch peeling for several eps, core numbers (Alg 3), level-round count (core_decomp_loop) and the
   kmax-core density. They are stored as ``<name>.npz``.

Usage: ``python tests/golden/make_golden.py`` (needs the reference tree: $GA_REFERENCE_ROOT, else /root/reference;
the outputs are committed).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import Reference  # noqa: E402
from oracle.build_oracle import REF_ROOT  # noqa: E402

REF_SCRIPTS = os.path.join(REF_ROOT, "scripts")
FIXTURES = [
    ("t_er300", "gen_test_graph.py", ["300", "0.05", "1"]),
    ("t_er800", "gen_test_graph.py", ["800", "0.02", "7"]),
    ("t_pl400", "gen_powerlaw.py", ["400", "4", "3"]),
    ("t_pl900", "gen_powerlaw.py", ["900", "6", "5"]),
]
EPS = [(1, 10), (1, 1), (0, 1), (3, 7), (1, 20), (1, 2)]


def main() -> None:
    ref = Reference()
    summary = {}
    for name, script, args in FIXTURES:
        path = os.path.join(HERE, name + ".txt")
        out = subprocess.check_output([sys.executable, os.path.join(REF_SCRIPTS, script), *args, path], text=True)
        brute = int(out.strip().splitlines()[-1])
        g = ref.load_graph(path)
        T = ref.triangles_serial(g)
        assert T == brute, (name, T, brute)
        Ts, sup = ref.edge_support(g)
        Td, deg = ref.triangle_degrees(g)
        core, kmax = ref.core_decomposition(g)
        core_l, kmax_l, rounds = ref.core_levels(g)
        assert (core_l == core).all() and kmax_l == kmax
        knum, kden = ref.core_level_density(g, core, kmax)
        arrays = dict(rowptr=g.rowptr, col=g.col, src=g.src, sup=sup, deg=deg, core=core)
        peel = {}
        for num, den in EPS:
            p = ref.batch_peel(g, num, den)
            assert p.ok
            arrays[f"removed_round_{num}_{den}"] = p.removed_round
            peel[f"{num}/{den}"] = dict(best_num=p.best_num, best_den=p.best_den, best_round=p.best_round,
                                         rounds=p.rounds)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        summary[name] = dict(generator=f"{script} {' '.join(args)}", brute_force_triangles=brute, n=g.n, m=g.m,
                             max_out_degree=g.max_out_degree, triangles=T, kmax=kmax, core_rounds=rounds,
                             kmax_core_density=[knum, kden], peel=peel)
        print(name, summary[name]["n"], summary[name]["m"], T, kmax, rounds)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(summary, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
