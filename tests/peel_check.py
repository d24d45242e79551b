"""The reference's removed_round check (emu_densest.cpp:44-54,153-166), restated: from the graph and a peeling's
removed_round array alone, recompute each round's alive count and triangle count and the best round (the first
strictly denser one, peel_improves densest.h:76-78), independently of the loop that produced them."""
from __future__ import annotations

import numpy as np

from test_dsg import triangles_of

NEVER = 0xFFFFFFFF


def best_from_removed_round(g, removed_round: np.ndarray) -> tuple[int, int, int, int]:
    """(best_num, best_den, best_round, rounds) implied by removed_round. Like the reference's check
    (emu_densest.cpp:153), every vertex must have been removed in some round: a loop that stopped early fails here
    instead of passing with never-removed vertices read as alive for ever."""
    rr = removed_round.astype(np.int64)
    assert not (rr == NEVER).any(), f"{int((rr == NEVER).sum())} vertices never removed"
    rounds = int(rr.max()) + 1 if rr.size else 0
    tris = triangles_of(g)
    # a triangle lives while all its corners do: it leaves in the round its first corner leaves
    gone = np.minimum(np.minimum(rr[tris[:, 0]], rr[tris[:, 1]]), rr[tris[:, 2]]) if len(tris) else np.zeros(0)
    best = (0, 0, 0)
    for r in range(rounds):
        nalive = int((rr >= r).sum())
        T = int((gone >= r).sum())
        if best[1] == 0 or T * best[1] > best[0] * nalive:
            best = (T, nalive, r)
    return best[0], best[1], best[2], rounds
