"""Shared fixtures. `gpu`-marked tests need a CUDA device and call the product through its C ABI; the rest run on CPU.

The checker libraries (oracle/liboracle.so, and oracle/_ref/libga_ref.so where the reference sources exist or the
built file was shipped) are built on demand; the product library must have been built (``__graft_entry__.build()``).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = ["t_er300", "t_er800", "t_pl400", "t_pl900"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference
    try:
        return Reference()
    except (FileNotFoundError, OSError) as e:
        pytest.skip(f"reference build unavailable: {e}")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def golden_arrays(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def fixture_path(name: str) -> str:
    return os.path.join(GOLDEN, name + ".txt")


@pytest.fixture(scope="session")
def ga():
    import graph_analyzer_b200 as ga_mod
    ga_mod.lib()
    return ga_mod


@pytest.fixture(scope="session")
def cuda_ok(ga):
    if ga.device_count() == 0:
        pytest.skip("no CUDA device")
    return True


def random_pairs(rng: np.random.Generator, n: int, p: float) -> np.ndarray:
    """Erdos-Renyi pairs (u < v) on n vertices."""
    iu, iv = np.triu_indices(n, 1)
    keep = rng.random(iu.size) < p
    return np.stack([iu[keep], iv[keep]], 1).astype(np.uint32)


def hub_pairs(rng: np.random.Generator, hubs: int, leaves: int, cluster: int) -> tuple[int, np.ndarray]:
    """Hub graphs in the style of the reference's --hub suite (emu_dsg.cpp:654-696): hubs with 40-100+ leaf
    neighbours and a few links into a dense cluster, ids shuffled."""
    n = hubs + leaves + cluster
    perm = rng.permutation(n)
    e = []
    c0 = hubs + leaves
    for a in range(c0, n):
        for b in range(a + 1, n):
            if rng.random() < 0.7:
                e.append((a, b))
    for h in range(hubs):
        for leaf in range(leaves):
            if rng.random() < 0.9:
                e.append((hubs + leaf, h))
        for _ in range(2 + rng.integers(3)):
            e.append((h, c0 + rng.integers(cluster)))
        for h2 in range(h + 1, hubs):
            e.append((h, h2))
    p = np.array([(perm[a], perm[b]) for a, b in e], dtype=np.uint32).reshape(-1, 2)
    return n, p
