"""GPU tests of the batched forms: a window of update batches applied by
gv_batch_run must leave exactly the graph that applying the batches one by
one leaves (the oracle applies them one by one); batched PPR queries must
match the oracle per query; the autotuner must return a valid config."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_same_adjacency, assert_sound, make_graph, rmat_graph, sample_existing

gv_b200 = pytest.importorskip("gv_b200")
pytestmark = pytest.mark.gpu

PR_L1 = 1e-6
HUB_PR_L1 = 1e-5  # fp32 floor of a graph with a 7000-entry hub row (see its test)


def _window(n, off, dst, rng, nb=12):
    """Batches that overlap on purpose: pairs inserted, deleted, re-inserted
    across batches, duplicates, self-loops."""
    batches = []
    pool_s, pool_d = gv_b200.gen_uniform(n, 4000, seed=int(rng.integers(1 << 30)))
    for b in range(nb):
        k = int(rng.integers(50, 800))
        ins = rng.integers(0, len(pool_s), k)
        ins_s, ins_d = pool_s[ins], pool_d[ins]
        es, ed = sample_existing(off, dst, int(rng.integers(20, 400)), rng)
        # delete some of the shared pool too, so later batches re-insert them
        dl = rng.integers(0, len(pool_s), int(rng.integers(10, 300)))
        del_s = np.concatenate([es, pool_s[dl]])
        del_d = np.concatenate([ed, pool_d[dl]])
        loops = rng.integers(0, n, 5).astype(np.uint32)
        ins_s = np.concatenate([ins_s, loops, ins_s[:10]])
        ins_d = np.concatenate([ins_d, loops, ins_d[:10]])
        batches.append((ins_s.astype(np.uint32), ins_d.astype(np.uint32), del_s.astype(np.uint32),
                        del_d.astype(np.uint32)))
    return batches


@pytest.mark.parametrize("graph_mode,device_inputs", [(False, False), (True, False), (False, True)])
def test_window_equals_sequential(graph_mode, device_inputs):
    import torch
    scale = 11
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=3)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    off, dst, _ = o.export()
    batches = _window(n, off, dst, np.random.default_rng(11))
    g = make_graph(n)
    g.batch_insert(s, d)
    if device_inputs:
        descs, srcs, dsts, p = [], [], [], 0
        for a, b, c, e in batches:
            descs.append((p, len(a), len(c)))
            srcs += [a, c]
            dsts += [b, e]
            p += len(a) + len(c)
        src = torch.from_numpy(np.concatenate(srcs).view(np.int32)).cuda()
        dstt = torch.from_numpy(np.concatenate(dsts).view(np.int32)).cuda()
        g.batch_run((descs, src, dstt), compact=True, graph=graph_mode)
    else:
        g.batch_run(batches, compact=True, graph=graph_mode)
    g.synchronize()
    for ins_s, ins_d, del_s, del_d in batches:
        o.insert(ins_s, ins_d)
        o.delete(del_s, del_d)
    assert_same_adjacency(g, o)
    assert_sound(g)


def test_window_graph_is_captured_once_and_replayed():
    """Windows of the same capacity replay one captured graph (sizes are read
    on the device); every window leaves the graph the oracle's sequential
    application leaves."""
    scale = 11
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=13)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    g = make_graph(n)
    g.batch_insert(s, d)
    rng = np.random.default_rng(21)
    for w in range(4):
        off, dst, _ = o.export()
        batches = _window(n, off, dst, rng, nb=int(rng.integers(3, 10)))
        g.batch_run(batches, compact=True, graph=True)
        g.synchronize()
        for ins_s, ins_d, del_s, del_d in batches:
            o.insert(ins_s, ins_d)
            o.delete(del_s, del_d)
        assert_same_adjacency(g, o)
        assert_sound(g)
    assert g.last_stat("window_persistent") == 4
    assert g.last_stat("window_captures") == 1
    assert g.last_stat("window_replays") == 3


def test_window_hub_segments_and_mixed_operations():
    """Segments above the lane-group limits (a hub with more than 64 blocks of
    32 entries, a window putting thousands of entries on one vertex) go to
    whole CTAs of the persistent launch; inserts and deletes of the same
    vertex in one segment."""
    n = 1 << 14
    rng = np.random.default_rng(3)
    others = np.setdiff1d(np.arange(n, dtype=np.uint32), [7, 11])
    h7 = rng.permutation(others)[:6000]  # 188 blocks of 32
    bs, bd = rmat_graph(14, 4, seed=3)
    s = np.concatenate([np.full(len(h7), 7, np.uint32), bs])
    d = np.concatenate([h7, bd])
    g = make_graph(n, block_size=32, threads_per_vertex=8)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    batches = []
    for b in range(6):
        ins_d = rng.permutation(others)[:1500].astype(np.uint32)   # new and existing neighbours of 7
        del_d = rng.choice(h7, 800, replace=False).astype(np.uint32)
        hub11 = rng.permutation(others)[:3000].astype(np.uint32)    # a vertex that becomes a hub in the window
        batches.append((np.concatenate([np.full(1500, 7, np.uint32), np.full(3000, 11, np.uint32)]),
                        np.concatenate([ins_d, hub11]),
                        np.concatenate([del_d, np.full(100, 11, np.uint32)]),
                        np.concatenate([np.full(800, 7, np.uint32), hub11[:100]])))
    g.batch_run(batches, compact=True)
    g.synchronize()
    for ins_s, ins_d, del_s, del_d in batches:
        o.insert(ins_s, ins_d)
        o.delete(del_s, del_d)
    assert_same_adjacency(g, o)
    assert_sound(g)
    assert g.last_stat("window_persistent") == 1


def test_window_exact_path_when_the_pool_is_tight():
    """A pool too small for the persistent path's worst case takes the
    two-stage path, which still applies a window that fits and rejects one
    that does not, whole."""
    n = 1 << 10
    s, d = rmat_graph(10, 4, seed=9)
    probe = make_graph(n, block_size=32, pool_blocks=1 << 14)
    probe.batch_insert(s, d)
    cap, free = probe.pool_stats()
    used = cap - free
    probe.close()
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    rng = np.random.default_rng(4)
    off, dst, _ = o.export()
    batches = _window(n, off, dst, rng, nb=1)
    # one block short of the window's worst case (one block per 32 of its
    # directed entries plus one per touched vertex), which is more than the
    # blocks it really needs
    E = 2 * sum(len(a) + len(c) for a, b, c, e in batches)
    worst = (E + 31) // 32 + min(E, n)
    g = make_graph(n, block_size=32, pool_blocks=used + worst - 1)
    g.batch_insert(s, d)
    g.synchronize()
    assert g.pool_stats()[1] == worst - 1
    g.batch_run(batches, compact=True)
    g.synchronize()
    for ins_s, ins_d, del_s, del_d in batches:
        o.insert(ins_s, ins_d)
        o.delete(del_s, del_d)
    assert_same_adjacency(g, o)
    assert g.last_stat("window_exact") >= 1
    # a window far beyond the free blocks is rejected and leaves the graph as it was
    before = g.export_csr()
    big_s, big_d = gv_b200.gen_uniform(n, 200_000, seed=5)
    g.batch_run([(big_s, big_d, big_s[:0], big_d[:0])], compact=True)
    with pytest.raises(gv_b200.GvError):
        g.synchronize()
    after = g.export_csr()
    assert np.array_equal(before[0], after[0])
    assert_sound(g)


@pytest.mark.parametrize("graph_mode", [True, False])
def test_window_with_ppr_queries(graph_mode):
    """gv_batch_run_ppr: windows of updates followed by PPR queries on the
    graph they leave, as one unit (one replayed CUDA graph in graph mode);
    each window's graph against the oracle, each query against the oracle's
    PPR at the same sweep count; hubs large enough to be cut into items."""
    n = 1 << 12
    rng = np.random.default_rng(41)
    s, d = rmat_graph(12, 8, seed=41)
    others = np.setdiff1d(np.arange(n, dtype=np.uint32), [5])
    hub = rng.permutation(others)[:2500]       # 79 blocks of 32: several items
    s = np.concatenate([s, np.full(len(hub), 5, np.uint32)])
    d = np.concatenate([d, hub])
    g = make_graph(n, block_size=32, threads_per_vertex=8)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    for w in range(3):
        off, dst, _ = o.export()
        batches = _window(n, off, dst, rng, nb=4)
        sources = np.concatenate([[5], rng.choice(n, 11, replace=False)]).astype(np.uint32)
        x, sweeps = g.batch_run_ppr(batches, sources, compact=True, graph=graph_mode, max_iter=60)
        for ins_s, ins_d, del_s, del_d in batches:
            o.insert(ins_s, ins_d)
            o.delete(del_s, del_d)
        assert_same_adjacency(g, o)
        assert 0 < sweeps <= 60
        for j, src in enumerate(sources):
            xo, _ = o.ppr(int(src), 0.85, 1e-6, 60, fixed_sweeps=sweeps)
            assert np.abs(x[:, j].astype(np.float64) - xo).sum() < PR_L1, (w, j)
    # queries alone (no batches)
    x, sweeps = g.batch_run_ppr([], np.array([5, 17], np.uint32), graph=graph_mode, max_iter=60)
    xo, _ = o.ppr(17, 0.85, 1e-6, 60, fixed_sweeps=sweeps)
    assert np.abs(x[:, 1].astype(np.float64) - xo).sum() < PR_L1
    if graph_mode:
        assert g.last_stat("window_replays") >= 2
    g.close()


def test_window_rejects_bad_ids_whole():
    import torch
    n = 512
    s, d = rmat_graph(9, 8, seed=5)
    g = make_graph(n)
    g.batch_insert(s, d)
    g.synchronize()
    before = g.export_csr()
    src = torch.tensor([1, 2, 3, 4000], dtype=torch.int32, device="cuda")
    dst = torch.tensor([5, 6, 7, 8], dtype=torch.int32, device="cuda")
    g.batch_run(([(0, 2, 2)], src, dst), compact=True)
    with pytest.raises(gv_b200.GvError):
        g.synchronize()
    after = g.export_csr()
    assert np.array_equal(before[0], after[0]) and np.array_equal(np.sort(before[1]), np.sort(after[1]))
    assert_sound(g)


def test_ppr_batch_matches_oracle_per_query():
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=8)
    g = make_graph(n)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    sources = np.random.default_rng(2).choice(n, 24, replace=False).astype(np.uint32)
    x, sweeps = g.ppr_batch(sources, 0.85, 1e-6, 100)
    assert x.shape == (n, len(sources))
    for j, src in enumerate(sources):
        xo, _ = o.ppr(int(src), 0.85, 1e-6, 100, fixed_sweeps=sweeps)
        assert np.abs(x[:, j] - xo).sum() < PR_L1, j


@pytest.fixture(scope="module")
def hub_graph13():
    """R-MAT scale 13 plus a hub of 7000 entries (cut into several items),
    isolated vertices, and tombstones left by a delete batch."""
    n = 1 << 13
    rng = np.random.default_rng(41)
    s, d = rmat_graph(13, 8, seed=41)
    hub_d = rng.choice(np.arange(1, n, dtype=np.uint32), 7000, replace=False).astype(np.uint32)
    s = np.concatenate([s, np.zeros(7000, np.uint32)])
    d = np.concatenate([d, hub_d])
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    off, dst, _ = o.export()
    es, ed = sample_existing(off, dst, 2000, rng)
    o.delete(es, ed)
    return n, s, d, es, ed, o


@pytest.mark.parametrize("k", [1, 2, 3, 8, 13, 16, 24, 32])
@pytest.mark.parametrize("plan", ["1", "0"])
def test_ppr_batch_plan_and_store_match_oracle(hub_graph13, k, plan, monkeypatch):
    """Batched PPR over the sweep plan (default; strides 2 to 32, the
    single-vector sweep for one query) and over the store (GV_PR_PLAN=0):
    sources that are the hub, leaves, isolated vertices and a repeated
    source, per query against the oracle.  Twenty sweeps exactly (epsilon
    0): with epsilon 1e-6 some queries on this graph reach the fp32 floor of
    the residual and run to max_iter, where the iterate only drifts with
    rounding.  The tolerance is the fp32 floor of this graph: the hub's value
    (about 0.2) is a sum over 7000 entries, whose rounding alone gives an L1
    of 1e-6 to 7e-6 against the fp64 oracle, whatever the summation order
    (the store sweep shows 6.9e-6 on the query from vertex 191)."""
    import torch
    monkeypatch.setenv("GV_PR_PLAN", plan)
    n, s, d, es, ed, o = hub_graph13
    g = make_graph(n, threads_per_vertex=8)
    g.batch_insert(s, d)
    g.batch_delete(es, ed)  # tombstones stay: the plan maps them to its sentinel
    deg = g.degrees()
    assert deg[0] > 3 * 2048 and (deg == 0).any()
    rng = np.random.default_rng(k)
    pick = [0, int(np.nonzero(deg == 0)[0][0]), int(np.nonzero(deg == 1)[0][0])]
    pick += list(rng.choice(n, 32, replace=False))
    sources = np.array((pick[:k - 1] + [pick[0]])[:k] if k > 3 else pick[:k], np.uint32)
    x, sweeps = g.ppr_batch(sources, 0.85, 0.0, 20)
    assert sweeps == 20
    for j, src in enumerate(sources):
        xo, _ = o.ppr(int(src), 0.85, 0.0, 20, fixed_sweeps=20)
        assert np.abs(x[:, j].astype(np.float64) - xo).sum() < HUB_PR_L1, (j, int(src))
    # device sources and output: the same values
    xd = torch.empty((n, k), dtype=torch.float32, device="cuda")
    _, sweeps_d = g.ppr_batch(sources, 0.85, 0.0, 20, out=xd)
    assert sweeps_d == sweeps
    assert np.array_equal(xd.cpu().numpy(), x)
    g.close()


def test_autotune_returns_a_candidate():
    scale = 10
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=4)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    off, dst, _ = o.export()
    batches = _window(n, off, dst, np.random.default_rng(5), nb=4)
    best, results = gv_b200.autotune(n, s, d, batches, hbm_budget_bytes=256 << 20)
    assert len(results) == 12
    assert best["block_size"] in (32, 64, 128) and best["threads_per_vertex"] in (4, 8, 16, 32)
    assert all(r["update_ms"] > 0 and r["pagerank_ms"] > 0 for r in results)
