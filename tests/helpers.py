"""Shared helpers for the parity tests (inputs, comparisons)."""
from __future__ import annotations

import numpy as np

import oracle


TEST_BUDGET = 2 << 30  # bytes of HBM per test graph (keeps the device mostly free)


def make_graph(n: int, **kw):
    """A libgv graph with a modest HBM budget unless the test sets one."""
    import gv_b200
    if "pool_blocks" not in kw and "hbm_budget_bytes" not in kw:
        kw["hbm_budget_bytes"] = TEST_BUDGET
    return gv_b200.GraphVine(n, **kw)


def rmat_graph(scale: int, edge_factor: int, seed: int):
    """Seeded R-MAT pairs (the generator libgv and the oracle share)."""
    return oracle.rmat_pairs(scale, edge_factor << scale, seed)


def sorted_adjacency(off, dst, w=None):
    """Per-vertex sorted neighbour arrays (and aligned weights)."""
    n = len(off) - 1
    out_d = np.empty_like(dst)
    out_w = None if w is None else np.empty_like(w)
    for u in range(n):
        a, b = int(off[u]), int(off[u + 1])
        if b - a:
            o = np.argsort(dst[a:b], kind="stable")
            out_d[a:b] = dst[a:b][o]
            if w is not None:
                out_w[a:b] = w[a:b][o]
    return out_d, out_w


def assert_same_adjacency(gv_graph, ora: oracle.OracleGraph, weights: bool = False):
    off, dst, w = gv_graph.export_csr(with_weights=weights)
    ooff, odst, ow = ora.export()
    assert np.array_equal(off, ooff), "per-vertex degrees differ"
    sd, sw = sorted_adjacency(off, dst, w)
    assert np.array_equal(sd, odst), "neighbour sets differ"
    if weights:
        assert np.array_equal(sw, ow), "weights differ"


def assert_sound(gv_graph):
    v, code, vert = gv_graph.check()
    assert v == 0, f"{v} invariant violations, first code {code} at {vert}"


def sample_existing(off, dst, k, rng, src_side=None):
    """k existing (u, v) entries sampled uniformly from a CSR snapshot."""
    m = len(dst)
    idx = rng.integers(0, m, size=k)
    src = np.searchsorted(off, idx, side="right").astype(np.int64) - 1
    return src.astype(np.uint32), dst[idx].astype(np.uint32)
