"""The full-size workloads' inputs, regenerated bit for bit from their seeds by the library's host generators (the
same parameters as bench.py's workloads): the Holme-Kim n = 1.70M graph, the R-MAT scale 22 graph and the 4,096-graph
Holme-Kim batch. Shared by make_fullsize.py (which records the reference's outputs on them) and the full-size GPU
tests (which compare the device results with those records)."""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

import graph_analyzer_b200 as ga  # noqa: E402

SEED = 1
HK = dict(n=1_700_000, m_lo=6, m_hi=7, p_hi=0.54, triad_p=0.3)
RMAT = dict(scale=22, edge_factor=8.52, abc=(0.57, 0.19, 0.19))
BATCH = dict(graphs=4096, n_lo=64, n_hi=262144, deg_lo=4.0, deg_hi=32.0, p_lo=0.1, p_hi=0.7)


def sha(a: np.ndarray) -> str:
    """SHA-256 of an array's bytes (uint32 arrays: little-endian words)."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def hk_graph() -> ga.Graph:
    return ga.graph_from_pairs(HK["n"], ga.gen_holme_kim(HK["n"], HK["m_lo"], HK["m_hi"], HK["p_hi"], HK["triad_p"],
                                                         seed=SEED))


def rmat_graph() -> ga.Graph:
    s = RMAT["scale"]
    return ga.graph_from_pairs(1 << s, ga.gen_rmat(s, int(RMAT["edge_factor"] * (1 << s)), *RMAT["abc"], seed=SEED))


def batch_graphs() -> ga.HostBatch:
    b = BATCH
    return ga.gen_holme_kim_batch(b["graphs"], b["n_lo"], b["n_hi"], b["deg_lo"], b["deg_hi"], b["p_lo"], b["p_hi"],
                                  seed=SEED)
