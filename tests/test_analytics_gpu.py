"""GPU parity tests of the analytics against the fp64 / exact oracle.

Tolerances (stated per result):
  PageRank, PPR: fp32 result within 1e-6 L1 of the fp64 oracle run for the
                 same number of sweeps;
  TC:            bit-exact per vertex (uint64);
  BFS sigma:     exact uint64; BC fp32 within 1e-5 max-relative of fp64;
  weighted PR:   forward within 1e-6 L1; gradient within 1e-4 relative
                 (scaled by the largest entry) of the fp64 oracle.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_same_adjacency, make_graph, rmat_graph, sample_existing

gv_b200 = pytest.importorskip("gv_b200")
pytestmark = pytest.mark.gpu

PR_L1 = 1e-6
BC_REL = 1e-5


@pytest.fixture(scope="module")
def graph12():
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=21)
    g = make_graph(n, threads_per_vertex=8)
    g.batch_insert(s, d)
    g.synchronize()
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    return n, g, o


def test_pagerank_matches_oracle(graph12):
    n, g, o = graph12
    x, sweeps = g.static_pagerank(0.85, 1e-6, 100)
    xo, so = o.pagerank(0.85, 1e-6, 100, fixed_sweeps=sweeps)
    err = np.abs(x.astype(np.float64) - xo).sum()
    print(f"pagerank sweeps={sweeps} oracle_free_sweeps={o.pagerank(0.85, 1e-6, 100)[1]} L1={err:.3e}")
    assert err < PR_L1
    assert abs(sweeps - o.pagerank(0.85, 1e-6, 100)[1]) <= 1


@pytest.mark.parametrize("plan", ["1", "0"])
def test_pagerank_plan_and_store_sweeps_match_oracle(plan, monkeypatch):
    """The degree-ordered sweep plan (default) and the store sweep
    (GV_PR_PLAN=0) on a graph with every tier: isolated vertices, rows below
    8, 64 and 2048 entries, and hubs cut into several items; static,
    warm-started and personalised runs against the oracle."""
    monkeypatch.setenv("GV_PR_PLAN", plan)
    n = 1 << 13
    rng = np.random.default_rng(31)
    s, d = rmat_graph(13, 8, seed=31)
    hub = np.full(7000, 3, np.uint32)
    hub_d = rng.choice(np.setdiff1d(np.arange(n, dtype=np.uint32), [3]), 7000, replace=False).astype(np.uint32)
    s = np.concatenate([s, hub])
    d = np.concatenate([d, hub_d])
    g = make_graph(n, threads_per_vertex=8)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    deg = g.degrees()
    assert (deg == 0).any() and deg.max() > 3 * 2048
    x, sweeps = g.static_pagerank(0.85, 1e-6, 100)
    xo, _ = o.pagerank(0.85, 1e-6, 100, fixed_sweeps=sweeps)
    assert np.abs(x.astype(np.float64) - xo).sum() < PR_L1
    # warm start after a batch: the same fixed point
    ins_s, ins_d = gv_b200.gen_uniform(n, 3000, seed=8)
    g.batch_insert(ins_s, ins_d)
    o.insert(ins_s, ins_d)
    xd, sd = g.dynamic_pagerank(x, 0.85, 1e-6, 100)
    xod, _ = o.pagerank(0.85, 1e-6, 100, x_init=x.astype(np.float64), fixed_sweeps=sd)
    assert np.abs(xd.astype(np.float64) - xod).sum() < PR_L1
    # personalised from the hub and from a leaf
    for src in (3, int(np.nonzero(deg == 1)[0][0])):
        xp, sp = g.ppr(src, 0.85, 1e-6, 100)
        xop, _ = o.ppr(src, 0.85, 1e-6, 100, fixed_sweeps=sp)
        assert np.abs(xp.astype(np.float64) - xop).sum() < PR_L1
    g.close()


def test_pagerank_fixed_sweeps_and_tombstones(graph12):
    n, _, _ = graph12
    s, d = rmat_graph(12, 16, seed=21)
    g = make_graph(n, block_size=32, threads_per_vertex=4)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    off, dst, _ = o.export()
    es, ed = sample_existing(off, dst, 3000, np.random.default_rng(4))
    g.batch_delete(es, ed)  # tombstones stay until compaction; PageRank skips them
    o.delete(es, ed)
    g.synchronize()
    x, sweeps = g.static_pagerank(0.85, 0.0, 20)
    assert sweeps == 20
    xo, _ = o.pagerank(0.85, 0.0, 20, fixed_sweeps=20)
    assert np.abs(x - xo).sum() < PR_L1


def test_dynamic_pagerank_reaches_static_fixed_point(graph12):
    n, _, _ = graph12
    s, d = rmat_graph(12, 16, seed=21)
    g = make_graph(n)
    g.batch_insert(s, d)
    x0, sw0 = g.static_pagerank(0.85, 1e-6, 200)
    ui, vi = gv_b200.gen_uniform(n, 300, seed=3)
    g.batch_insert(ui, vi)
    g.synchronize()
    xs, sws = g.static_pagerank(0.85, 1e-6, 200)
    xd, swd = g.dynamic_pagerank(x0, 0.85, 1e-6, 200)
    # both stop within eps of the same fixed point: |x - x*| <= eps * alpha / (1 - alpha)
    print(f"static sweeps={sws} warm-start sweeps={swd} L1(static,dynamic)={np.abs(xs - xd).sum():.3e}")
    assert swd < 200
    assert np.abs(xs - xd).sum() < 2 * 1e-6 * 0.85 / 0.15


def test_ppr_matches_oracle(graph12):
    n, g, o = graph12
    src = 5
    x, sweeps = g.ppr(src, 0.85, 1e-6, 100)
    xo, _ = o.ppr(src, 0.85, 1e-6, 100, fixed_sweeps=sweeps)
    assert np.abs(x - xo).sum() < PR_L1


@pytest.mark.parametrize("tpv", [4, 16])
def test_triangle_count_bit_exact(tpv):
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=31)
    g = make_graph(n, threads_per_vertex=tpv)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    pv, tot = g.static_tc()
    opv, otot = o.tc()
    assert tot == otot
    assert np.array_equal(pv, opv)
    # after deletes (tombstones) and compaction
    off, dst, _ = o.export()
    es, ed = sample_existing(off, dst, 5000, np.random.default_rng(7))
    g.batch_delete(es, ed)
    o.delete(es, ed)
    pv, tot = g.static_tc()
    assert np.array_equal(pv, o.tc()[0])
    g.compaction()
    pv, tot = g.static_tc()
    assert np.array_equal(pv, o.tc()[0])


def test_triangle_subset_incident(graph12):
    n, g, o = graph12
    sub = np.random.default_rng(1).choice(n, 300, replace=False).astype(np.uint32)
    assert np.array_equal(g.tc_subset(sub), o.tc_incident(sub))


@pytest.mark.parametrize("packed", ["0", "1"])
def test_hub_triangles_use_cta_sort(packed, monkeypatch):
    # a 1100-clique: its lowest-ranked member has an oriented list of 1099
    # entries, above the 1024-entry warp sort, so the CTA sort runs (merge
    # path) or one CTA takes the vertex (packed path)
    monkeypatch.setenv("GV_TC_PACKED", packed)
    n = 1 << 13
    K = 1100
    iu, ju = np.triu_indices(K, 1)
    perm = np.random.default_rng(5).permutation(n)[:K].astype(np.uint32)
    rs, rd = rmat_graph(13, 4, seed=8)
    s = np.concatenate([perm[iu], rs])
    d = np.concatenate([perm[ju], rd])
    g = make_graph(n)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    pv, tot = g.static_tc()
    opv, otot = o.tc()
    assert tot == otot and np.array_equal(pv, opv)


def test_bfs_sigma_exact(graph12):
    n, g, o = graph12
    for src in (0, 17, 1000):
        dist, sigma = g.bfs_sigma(src)
        od, osg = o.bfs_sigma(src)
        assert np.array_equal(dist, od)
        assert np.array_equal(sigma, osg)


def test_bc_sampled_sources(graph12):
    n, g, o = graph12
    src = np.random.default_rng(3).choice(n, 64, replace=False).astype(np.uint32)
    b = g.bc(src)
    ob = o.bc(src)
    rel = np.max(np.abs(b - ob) / np.maximum(np.abs(ob), 1e-300) * (ob != 0))
    print(f"bc max relative error {rel:.3e}")
    assert rel < BC_REL
    assert np.all(b[ob == 0] == 0)


@pytest.mark.parametrize("count", [1, 31, 33, 63, 65, 100])
def test_bc_pass_widths(graph12, count):
    """Source counts that leave a 32-source pass, partial halves of a
    64-source pass, or both."""
    n, g, o = graph12
    src = np.random.default_rng(count).choice(n, count, replace=False).astype(np.uint32)
    b = g.bc(src)
    ob = o.bc(src)
    rel = np.max(np.abs(b - ob) / np.maximum(np.abs(ob), 1e-300) * (ob != 0))
    assert rel < BC_REL
    assert np.all(b[ob == 0] == 0)


def test_bc_pull_levels_give_the_same_scores(monkeypatch, graph12):
    """Forward levels by pull (GV_BC_PULL, from rarely to nearly always) or by
    push give the same path counts, so the scores are bit-for-bit equal."""
    n, g, o = graph12
    src = np.random.default_rng(12).choice(n, 64, replace=False).astype(np.uint32)
    monkeypatch.setenv("GV_BC_PULL", "0")
    ref = g.bc(src)
    for alpha in ("1", "2", "1000"):
        monkeypatch.setenv("GV_BC_PULL", alpha)
        assert np.array_equal(g.bc(src), ref), alpha
    ob = o.bc(src)
    rel = np.max(np.abs(ref - ob) / np.maximum(np.abs(ob), 1e-300) * (ob != 0))
    assert rel < BC_REL


def test_bc_multi_matches_single(graph12):
    """Requests paired into shared passes score as they do alone."""
    n, g, o = graph12
    rng = np.random.default_rng(8)
    reqs = [rng.choice(n, k, replace=False).astype(np.uint32) for k in (5, 32, 40, 1, 17)]
    reqs.append(np.array([7, 7, 300], np.uint32))  # a repeated source counts twice
    got = g.bc_multi(reqs)
    assert got.shape == (len(reqs), n)
    for r, src in enumerate(reqs):
        alone = g.bc(src)
        assert np.allclose(got[r], alone, rtol=1e-6, atol=0), r
        ob = o.bc(src)
        rel = np.max(np.abs(got[r] - ob) / np.maximum(np.abs(ob), 1e-300) * (ob != 0))
        assert rel < BC_REL, r
    again = g.bc_multi(reqs)
    assert np.array_equal(got, again)  # repeatable bit for bit


def test_bc_multi_every_vertex_and_rejects():
    scale = 9
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=13)
    g = make_graph(n)
    g.batch_insert(s, d)
    got = g.bc_multi([np.array([], np.uint32), np.array([3, 4], np.uint32)])
    assert np.allclose(got[0], g.bc(), rtol=1e-6, atol=0)
    assert np.allclose(got[1], g.bc(np.array([3, 4], np.uint32)), rtol=1e-6, atol=0)
    with pytest.raises(RuntimeError):
        g.bc_multi([np.array([n], np.uint32)])


def test_bc_all_sources_small():
    scale = 9
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=13)
    g = make_graph(n)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    b = g.bc()
    ob = o.bc()
    nz = ob != 0
    assert np.max(np.abs(b[nz] - ob[nz]) / ob[nz]) < BC_REL


def _weighted(scale, seed):
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=seed)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.1, 1.0, len(s)).astype(np.float32)
    g = make_graph(n, directed=True, weighted=True)
    g.batch_insert(s, d, w)
    o = oracle.OracleGraph(n, directed=True, weighted=True)
    o.insert(s, d, w)
    return n, g, o, rng


def test_wpr_forward_and_gradient():
    n, g, o, rng = _weighted(11, 41)
    x, sw = g.wpr_forward(0.85, 1e-9, 300)
    xo, _ = o.wpr_forward(0.85)
    assert np.abs(x - xo).sum() < PR_L1
    c = rng.standard_normal(n)
    lo, _ = o.wpr_adjoint(c)
    for mode in (0, 1):
        grad, lam, _ = g.wpr_backward(x, c.astype(np.float32), 0.85, 1e-9, 300, mode=mode)
        go = o.wpr_gradient(xo, lo, c, mode=mode)
        # align by (u, v): the GPU export order is storage order
        off, dst, _ = g.export_csr()
        ooff, odst, _ = o.export()
        assert np.array_equal(off, ooff)
        src = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
        key_g = src.astype(np.uint64) * n + dst
        key_o = src.astype(np.uint64) * n + odst
        gg = grad[np.argsort(key_g)]
        gref = go[np.argsort(key_o)]
        scale = np.abs(gref).max()
        err = np.abs(gg - gref).max() / scale
        print(f"mode {mode}: max |grad - fp64| / max|grad| = {err:.3e}")
        assert err < 1e-4


def test_wpr_gradient_matches_dense_fp64_gradient_scale12():
    """The differentiation workload's dense check: directed weighted R-MAT
    scale 12 (weights U(0.1, 1], normalised per row), the GPU's gradient of
    sum c_i x_i with respect to every raw weight against the gradient from
    dense fp64 solves of the forward and transposed systems (numpy)."""
    scale = 12
    n = 1 << scale
    rng = np.random.default_rng(1212)
    s, d = rmat_graph(scale, 16, seed=1212)
    w = (1.0 - 0.9 * rng.random(len(s))).astype(np.float32)
    g = make_graph(n, directed=True, weighted=True)
    g.batch_insert(s, d, w)
    g.synchronize()
    off, dst, wt = g.export_csr(with_weights=True)
    src = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
    W = np.zeros((n, n))
    W[src, dst] = wt.astype(np.float64)
    rs = W.sum(1)
    P = np.divide(W, rs[:, None], out=np.zeros_like(W), where=rs[:, None] > 0)
    a = 0.85
    x = np.linalg.solve(np.eye(n) - a * P.T, np.full(n, (1 - a) / n))
    c = rng.standard_normal(n)
    lam = np.linalg.solve(np.eye(n) - a * P, c)
    # d J / d raw w_uv = a x_u (lam_v - (P lam)_u) / s_u
    Plam = P @ lam
    want = a * x[src] * (lam[dst] - Plam[src]) / rs[src]
    xg, _ = g.wpr_forward(a, 1e-9, 300)
    assert np.abs(xg.astype(np.float64) - x).sum() < PR_L1
    grad, _, _ = g.wpr_backward(xg, c.astype(np.float32), a, 1e-9, 300, mode=0)
    err = np.abs(grad.astype(np.float64) - want).max() / np.abs(want).max()
    print(f"scale 12: {len(dst)} entries, max |grad - dense fp64| / max |grad| = {err:.3e}")
    assert err < 1e-4
    g.close()


@pytest.mark.parametrize("mode", ["local", "global", ""])
def test_triangle_subset_paths_agree(mode, monkeypatch):
    """Both subset paths (neighbour hash sets, whole-graph oriented count) are
    bit-exact; the graph has a hub above the shared-memory table (global
    table path), tombstones from deletes without compaction, and the subset
    repeats vertices."""
    scale = 14
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=31)
    rng = np.random.default_rng(3)
    hub = 77
    nb = rng.choice(n, 9000, replace=False).astype(np.uint32)
    nb = nb[nb != hub]
    s = np.concatenate([s, np.full(len(nb), hub, np.uint32)])
    d = np.concatenate([d, nb])
    g = make_graph(n)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    off, dst, _ = o.export()
    ds, dd = sample_existing(off, dst, 3000, rng)
    g.batch_delete(ds, dd)
    o.delete(ds, dd)
    sub = np.concatenate([[hub], rng.choice(n, 400), nb[:60], [hub]]).astype(np.uint32)
    if mode:
        monkeypatch.setenv("GV_TC_SUBSET", mode)
    got = g.tc_subset(sub)
    assert np.array_equal(got, o.tc_incident(sub))
    if mode == "local":
        assert g.last_stat("tc_subset_local") == 1
    elif mode == "global":
        assert g.last_stat("tc_subset_local") == 0


@pytest.mark.parametrize("packed", ["0", "1"])
def test_triangle_paths_total_only_and_incident(packed, monkeypatch, graph12):
    """Merge and packed paths, the total-only mode (no per-vertex output) and
    the incident counts of the whole-graph subset path all match the oracle."""
    n, g, o = graph12
    monkeypatch.setenv("GV_TC_PACKED", packed)
    pv, tot = g.static_tc()
    opv, otot = o.tc()
    assert tot == otot and np.array_equal(pv, opv)
    _, tot2 = g.static_tc(per_vertex=False)
    assert tot2 == otot
    monkeypatch.setenv("GV_TC_SUBSET", "global")
    sub = np.random.default_rng(11).choice(n, 500, replace=False).astype(np.uint32)
    assert np.array_equal(g.tc_subset(sub), o.tc_incident(sub))


@pytest.mark.parametrize("core", ["0", "64", "1000", "32768"])
def test_total_triangles_dense_core(core, monkeypatch, graph12):
    """Total-only counts with the dense-core bit probes: no core (every edge
    merged), a core of 64 or 1000 vertices (edges split between probes and
    merges) and the default bound (every vertex with an edge in the core)."""
    n, g, o = graph12
    monkeypatch.setenv("GV_TC_CORE", core)
    _, otot = o.tc()
    _, tot = g.static_tc(per_vertex=False)
    assert tot == otot
    probes, csize = g.last_stat("tc_probes"), g.last_stat("tc_core")
    if core == "0":
        assert probes == 0 and csize == 0
    else:
        assert probes > 0 and 0 < csize <= int(core)
    # after tombstones and compaction
    off, dst, _ = o.export()
    es, ed = sample_existing(off, dst, 3000, np.random.default_rng(int(core) + 1))
    g2 = make_graph(n)
    s0, d0 = rmat_graph(12, 16, seed=21)  # the pairs of graph12
    perm = np.random.default_rng(int(core) + 2).permutation(len(s0))
    for part in np.array_split(perm, 4):  # batches in shuffled order leave the lists unsorted
        g2.batch_insert(s0[part], d0[part])
    g2.batch_delete(es, ed)
    o2 = oracle.OracleGraph(n)
    o2.insert(s0, d0)
    o2.delete(es, ed)
    assert g2.static_tc(per_vertex=False)[1] == o2.tc()[1]
    g2.compaction()
    assert g2.static_tc(per_vertex=False)[1] == o2.tc()[1]
    g2.close()


def test_total_triangles_without_a_core():
    """30000 disjoint triangles: every vertex has degree 2, so no degree
    threshold leaves at most 65504 vertices above it and every edge takes
    the merge path; and an empty graph counts 0."""
    k = 30000
    n = 3 * k
    a = np.arange(k, dtype=np.uint32) * 3
    s = np.concatenate([a, a + 1, a + 2])
    d = np.concatenate([a + 1, a + 2, a])
    g = make_graph(n)
    g.batch_insert(s, d)
    assert g.static_tc(per_vertex=False)[1] == k
    assert g.last_stat("tc_core") == 0 and g.last_stat("tc_probes") == 0
    e = make_graph(64)
    assert e.static_tc(per_vertex=False)[1] == 0
    g.close()
    e.close()


def test_core_list_order_does_not_change_counts(monkeypatch, graph12):
    """The bank-spreading reorder of the core lists (GV_TC_COLOR) changes
    only the order in which entries are tested."""
    n, g, o = graph12
    monkeypatch.setenv("GV_TC_CORE", "1000")
    _, otot = o.tc()
    for color in ("0", "1"):
        monkeypatch.setenv("GV_TC_COLOR", color)
        assert g.static_tc(per_vertex=False)[1] == otot


def test_sweep_split_does_not_change_pagerank(monkeypatch, graph12):
    """The fused sweep's CTA shares per tier (GV_SWEEP_SPLIT) move work
    between CTAs, never between lanes: the ranks are bit-for-bit the same."""
    n, g, o = graph12
    ref, sw = g.static_pagerank(0.85, 1e-6, 100)
    for split in ("1,1,14", "8,4,4", "5,5,6"):
        monkeypatch.setenv("GV_SWEEP_SPLIT", split)
        x, sw2 = g.static_pagerank(0.85, 1e-6, 100)
        assert sw2 == sw and np.array_equal(x, ref), split


def test_total_triangles_core_with_hub_clique(monkeypatch):
    """A 1100-clique inside an R-MAT graph: the clique members form the core
    and their rows hold 1099-entry lists."""
    monkeypatch.setenv("GV_TC_CORE", "2048")
    n = 1 << 13
    K = 1100
    iu, ju = np.triu_indices(K, 1)
    perm = np.random.default_rng(6).permutation(n)[:K].astype(np.uint32)
    rs, rd = rmat_graph(13, 4, seed=9)
    s = np.concatenate([perm[iu], rs])
    d = np.concatenate([perm[ju], rd])
    g = make_graph(n)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    assert g.static_tc(per_vertex=False)[1] == o.tc()[1]
    assert g.last_stat("tc_core") > 0


def test_wpr_forward_hub_in_edges_and_repeatable():
    """A vertex with 3000 in-edges takes the CTA-per-vertex sweep; the sorted
    in-edge transpose makes two calls bit-for-bit equal."""
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=13)
    rng = np.random.default_rng(13)
    hs = rng.choice(n, 3000, replace=False).astype(np.uint32)
    hs = hs[hs != 5]
    s = np.concatenate([s, hs])
    d = np.concatenate([d, np.full(len(hs), 5, np.uint32)])
    w = rng.uniform(0.1, 1.0, len(s)).astype(np.float32)
    g = make_graph(n, directed=True, weighted=True)
    g.batch_insert(s, d, w)
    o = oracle.OracleGraph(n, directed=True, weighted=True)
    o.insert(s, d, w)
    x1, _ = g.wpr_forward(0.85, 1e-9, 300)
    x2, _ = g.wpr_forward(0.85, 1e-9, 300)
    xo, _ = o.wpr_forward(0.85)
    assert np.abs(x1 - xo).sum() < PR_L1
    assert np.array_equal(x1, x2)


def _mixed_batch(g, n, rng, n_new=3000, n_del=2000):
    """Inserts: new uniform pairs, duplicates, self-loops, pairs already in the
    graph; deletes: existing pairs, some of this batch's inserts, absent pairs."""
    off, dst, _ = g.export_csr()
    ins_s, ins_d = gv_b200.gen_uniform(n, n_new, seed=int(rng.integers(1 << 30)))
    es, ed = sample_existing(off, dst, 300, rng)
    loops = rng.integers(0, n, 40).astype(np.uint32)
    ins_s = np.concatenate([ins_s, ins_s[:100], es, loops])
    ins_d = np.concatenate([ins_d, ins_d[:100], ed, loops])
    ds, dd = sample_existing(off, dst, n_del, rng)
    absent_s, absent_d = gv_b200.gen_uniform(n, 100, seed=int(rng.integers(1 << 30)))
    del_s = np.concatenate([ds, ins_d[:150], absent_s, dd[:50]])
    del_d = np.concatenate([dd, ins_s[:150], absent_d, ds[:50]])
    return ins_s.astype(np.uint32), ins_d.astype(np.uint32), del_s.astype(np.uint32), del_d.astype(np.uint32)


@pytest.mark.parametrize("block,scale,ef", [(128, 12, 16), (32, 14, 8)])
def test_update_tc_deltas_are_exact(block, scale, ef):
    """gv_update_tc's total and per-vertex deltas equal the difference of two
    whole-graph counts, batch after batch, and the graph ends as the oracle's."""
    n = 1 << scale
    s, d = rmat_graph(scale, ef, seed=17)
    g = make_graph(n, block_size=block)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    rng = np.random.default_rng(23)
    pv0, t0 = g.static_tc()
    for _ in range(3):
        ins_s, ins_d, del_s, del_d = _mixed_batch(g, n, rng)
        dt, dpv = g.update_tc(ins_s, ins_d, del_s, del_d, per_vertex=True)
        o.insert(ins_s, ins_d)
        o.delete(del_s, del_d)
        pv1, t1 = g.static_tc()
        assert t1 == t0 + dt
        assert np.array_equal(pv1.astype(np.int64), pv0.astype(np.int64) + dpv)
        pv0, t0 = pv1, t1
    opv, otot = o.tc()
    assert otot == t0 and np.array_equal(opv, pv0)
    assert_same_adjacency(g, o)


def test_update_tc_rejects_bad_ids_and_keeps_graph():
    n = 1 << 10
    s, d = rmat_graph(10, 8, seed=3)
    g = make_graph(n)
    g.batch_insert(s, d)
    before = g.export_csr()
    with pytest.raises(gv_b200.GvError):
        g.update_tc(np.array([1, 2], np.uint32), np.array([3, 4], np.uint32),
                    np.array([5, n + 7], np.uint32), np.array([6, 1], np.uint32))
    after = g.export_csr()
    assert np.array_equal(before[0], after[0])


def test_pagerank_on_directed_store():
    """Directed stores run PageRank, PPR and the warm start over the sorted
    in-edge transpose; all match the oracle's directed PageRank."""
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=27)
    g = make_graph(n, directed=True)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n, directed=True)
    o.insert(s, d)
    x, sw = g.static_pagerank(0.85, 1e-6, 100)
    xo, _ = o.pagerank(0.85, 1e-6, 100, fixed_sweeps=sw)
    assert np.abs(x - xo).sum() < PR_L1
    xp, swp = g.ppr(5, 0.85, 1e-6, 100)
    xpo, _ = o.ppr(5, 0.85, 1e-6, 100, fixed_sweeps=swp)
    assert np.abs(xp - xpo).sum() < PR_L1
    xd, swd = g.dynamic_pagerank(x, 0.85, 1e-6, 100)
    xdo, _ = o.pagerank(0.85, 1e-6, 100, x_init=x.astype(np.float64), fixed_sweeps=swd)
    assert np.abs(xd - xdo).sum() < PR_L1
