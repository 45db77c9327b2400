"""GPU parity tests of the edge-block CBT store against the oracle:
bulk build, set-union insert, set-difference delete, compaction, the
structural invariants, and the error paths (pool exhaustion, bad ids)."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_same_adjacency, assert_sound, make_graph, rmat_graph, sample_existing

gv_b200 = pytest.importorskip("gv_b200")
pytestmark = pytest.mark.gpu


def build_pair(n, s, d, **kw):
    g = make_graph(n, **kw)
    g.batch_insert(s, d)
    g.synchronize()
    o = oracle.OracleGraph(n, directed=kw.get("directed", False), weighted=kw.get("weighted", False))
    o.insert(s, d)
    return g, o


@pytest.mark.parametrize("block,tpv", [(32, 4), (64, 8), (128, 8), (128, 32), (32, 16)])
def test_build_insert_delete_compact(block, tpv):
    scale = 10
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=1)
    g, o = build_pair(n, s, d, block_size=block, threads_per_vertex=tpv)
    assert g.num_edges() == o.num_edges()
    assert_same_adjacency(g, o)
    assert_sound(g)
    rng = np.random.default_rng(block + tpv)
    # inserts: uniform pairs plus duplicates, self-loops and existing edges
    ui, vi = gv_b200.gen_uniform(n, 3000, seed=5)
    off, dst, _ = o.export()
    es, ed = sample_existing(off, dst, 500, rng)
    loops = rng.integers(0, n, 100).astype(np.uint32)
    ins_s = np.concatenate([ui, es, loops, ui[:200]])
    ins_d = np.concatenate([vi, ed, loops, vi[:200]])
    g.batch_insert(ins_s, ins_d)
    o.insert(ins_s, ins_d)
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)
    # deletes: existing edges (both directions) plus absent pairs
    off, dst, _ = o.export()
    es, ed = sample_existing(off, dst, 4000, rng)
    xs, xd = gv_b200.gen_uniform(n, 300, seed=8)
    del_s, del_d = np.concatenate([es, xs]), np.concatenate([ed, xd])
    g.batch_delete(del_s, del_d)
    o.delete(del_s, del_d)
    g.synchronize()
    assert g.num_edges() == o.num_edges()
    assert_same_adjacency(g, o)
    assert_sound(g)
    cap, free0 = g.pool_stats()
    g.compaction()
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)
    _, free1 = g.pool_stats()
    assert free1 >= free0
    # re-insert after compaction
    g.batch_insert(del_s[:1000], del_d[:1000])
    o.insert(del_s[:1000], del_d[:1000])
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)


def test_hub_paths_and_block_multiples():
    # one hub far above the lane-group thresholds, vertices whose degree is an
    # exact multiple of the block size, and a vertex that loses every edge
    n = 1 << 14
    B = 32
    hub = np.full(9000, 7, np.uint32)
    hub_d = np.setdiff1d(np.arange(n, dtype=np.uint32), [7])[:9000]
    # vertices 100..109 get exactly 64 = 2 blocks of neighbours, none shared with the hub
    mult_s = np.repeat(np.arange(100, 110, dtype=np.uint32), 64) + 12000
    mult_d = (np.tile(np.arange(64, dtype=np.uint32), 10) + 13000)
    s = np.concatenate([hub, mult_s])
    d = np.concatenate([hub_d, mult_d])
    g, o = build_pair(n, s, d, block_size=B, threads_per_vertex=8)
    assert_same_adjacency(g, o)
    assert_sound(g)
    rng = np.random.default_rng(0)
    # delete a random half of the hub plus every edge of vertex 100
    pick = rng.choice(9000, 4500, replace=False)
    ds = np.concatenate([hub[pick], np.full(64, 12100, np.uint32)])
    dd = np.concatenate([hub_d[pick], mult_d[:64]])
    g.batch_delete(ds, dd)
    o.delete(ds, dd)
    g.compaction()
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)
    assert g.degrees()[12100] == 0
    # a big insert batch into the hub (CTA path of apply)
    add = np.setdiff1d(np.arange(n, dtype=np.uint32), [7])[9000:12000]
    g.batch_insert(np.full(len(add), 7, np.uint32), add)
    o.insert(np.full(len(add), 7, np.uint32), add)
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)


def test_hubs_beyond_one_block_table_window():
    """Hubs of more than 1024 blocks of 32 entries (the CTA-per-vertex
    membership and compaction paths walk their blocks in windows of 1024
    table entries) and of more than 2048 blocks (the BC kernels' table
    windows): insert, BC and PageRank across windows, deletes spread over
    every window, compaction that moves tail entries into earlier windows,
    then inserts into the compacted hub, each step against the oracle."""
    scale = 17
    n = 1 << scale
    B = 32
    rng = np.random.default_rng(17)
    bs, bd = rmat_graph(scale, 4, seed=17)
    others = np.setdiff1d(np.arange(n, dtype=np.uint32), [5, 9])
    h5 = rng.permutation(others)[:80_000]           # 2500 blocks
    h9 = rng.permutation(others)[:40_000]           # 1250 blocks
    s = np.concatenate([bs, np.full(len(h5), 5, np.uint32), np.full(len(h9), 9, np.uint32)])
    d = np.concatenate([bd, h5, h9])
    g, o = build_pair(n, s, d, block_size=B, threads_per_vertex=8)
    assert_same_adjacency(g, o)
    assert_sound(g)
    assert g.degrees()[5] > 2048 * B
    src = np.array([5, 9, 77, 1234], np.uint32)
    b = g.bc(src)
    ob = o.bc(src)
    nz = ob != 0
    assert np.max(np.abs(b[nz] - ob[nz]) / np.abs(ob[nz])) < 1e-5
    assert np.all(b[~nz] == 0)
    x, sweeps = g.static_pagerank(0.85, 1e-6, 100)
    xo, _ = o.pagerank(0.85, 1e-6, 100, fixed_sweeps=sweeps)
    assert np.abs(x - xo).sum() < 1e-6
    # delete 60% of each hub's entries (spread over every window) plus some background
    d5 = h5[rng.random(len(h5)) < 0.6]
    d9 = h9[rng.random(len(h9)) < 0.6]
    ooff, odst, _ = o.export()
    es, ed = sample_existing(ooff, odst, 20_000, rng)
    ds = np.concatenate([np.full(len(d5), 5, np.uint32), d9, es])
    dd = np.concatenate([d5, np.full(len(d9), 9, np.uint32), ed])  # hub 9 deleted from the other side
    g.batch_delete(ds, dd)
    o.delete(ds, dd)
    g.compaction()
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)
    # re-insert part of what was deleted plus new neighbours into the compacted hubs
    add = np.concatenate([d5[:15_000], rng.permutation(others)[:30_000]])
    g.batch_insert(np.full(len(add), 5, np.uint32), add)
    o.insert(np.full(len(add), 5, np.uint32), add)
    g.batch_insert(d9[:10_000], np.full(10_000, 9, np.uint32))
    o.insert(d9[:10_000], np.full(10_000, 9, np.uint32))
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)
    pv, tot = g.static_tc()
    opv, otot = o.tc()
    assert tot == otot and np.array_equal(pv, opv)
    g.close()


def test_directed_store():
    n = 1 << 10
    s, d = rmat_graph(10, 8, seed=4)
    g, o = build_pair(n, s, d, directed=True)
    assert_same_adjacency(g, o)
    g.batch_delete(s[:500], d[:500])
    o.delete(s[:500], d[:500])
    g.compaction()
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)


def test_weighted_first_occurrence_and_compaction():
    n = 1 << 9
    s, d = rmat_graph(9, 8, seed=2)
    rng = np.random.default_rng(1)
    w = rng.uniform(0.1, 1.0, len(s)).astype(np.float32)
    g = make_graph(n, directed=True, weighted=True)
    g.batch_insert(s, d, w)
    o = oracle.OracleGraph(n, directed=True, weighted=True)
    o.insert(s, d, w)
    g.synchronize()
    assert_same_adjacency(g, o, weights=True)
    # re-inserting existing pairs with new weights keeps the stored weight
    g.batch_insert(s[:100], d[:100], w[:100] + 5)
    o.insert(s[:100], d[:100], w[:100] + 5)
    g.batch_delete(s[100:600], d[100:600])
    o.delete(s[100:600], d[100:600])
    g.compaction()
    g.synchronize()
    assert_same_adjacency(g, o, weights=True)
    assert_sound(g)


def test_bulk_build_from_csr_matches_insert():
    n = 1 << 10
    s, d = rmat_graph(10, 8, seed=9)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    off, dst, _ = o.export()
    g = make_graph(n)
    g.bulk_build(off, dst)
    g.synchronize()
    assert_same_adjacency(g, o)
    assert_sound(g)


def test_empty_and_degenerate_batches():
    n = 256
    g = make_graph(n)
    g.batch_insert(np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    loops = np.arange(n, dtype=np.uint32)
    g.batch_insert(loops, loops)
    g.batch_delete(loops, loops)
    g.compaction()
    g.synchronize()
    assert g.num_edges() == 0
    assert_sound(g)


def test_pool_exhaustion_rejects_batch_and_keeps_graph():
    n = 1 << 10
    g = make_graph(n, block_size=32, pool_blocks=200)
    s = np.arange(0, 100, dtype=np.uint32)
    d = s + 1
    g.batch_insert(s, d)
    g.synchronize()
    before = g.export_csr()
    big_s = np.repeat(np.arange(300, 700, dtype=np.uint32), 2)
    big_d = np.arange(800, 1600, dtype=np.uint32) % n
    g.batch_insert(big_s, big_d)
    with pytest.raises(gv_b200.GvError) as e:
        g.synchronize()
    assert "NOMEM" in str(e.value)
    after = g.export_csr()
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
    assert_sound(g)


def test_bad_ids_rejected():
    import torch
    n = 64
    g = make_graph(n)
    with pytest.raises(gv_b200.GvError) as e:
        g.batch_insert(np.array([1, 70], np.uint32), np.array([2, 3], np.uint32))
    assert "INVALID" in str(e.value)
    # device-resident batch: checked on the device, whole batch rejected
    src = torch.tensor([1, 2, 99], dtype=torch.int32, device="cuda")
    dst = torch.tensor([5, 6, 7], dtype=torch.int32, device="cuda")
    g.batch_insert(src, dst)
    with pytest.raises(gv_b200.GvError):
        g.synchronize()
    assert g.num_edges() == 0
    g.synchronize()  # status was cleared


def test_affected_flags():
    n = 128
    g = make_graph(n)
    g.batch_insert(np.array([1, 2], np.uint32), np.array([3, 4], np.uint32))
    a = g.affected()
    assert set(np.nonzero(a)[0]) == {1, 2, 3, 4}
    g.clear_affected()
    assert g.affected().sum() == 0


@pytest.mark.parametrize("directed", [False, True])
def test_add_and_delete_vertices(directed):
    """Vertices added past the table's capacity take edges like any other;
    deleting vertices removes exactly their incident edges; analytics run on
    the grown graph."""
    n0, k = 1000, 1500
    s, d = rmat_graph(10, 8, seed=12)
    s, d = s % n0, d % n0
    g = make_graph(n0, directed=directed)
    g.batch_insert(s, d)
    first = g.add_vertices(k)
    assert first == n0 and g.n == n0 + k
    n = n0 + k
    rng = np.random.default_rng(4)
    ns = rng.integers(0, n, 6000).astype(np.uint32)
    nd = rng.integers(n0, n, 6000).astype(np.uint32)
    g.batch_insert(ns, nd)
    o = oracle.OracleGraph(n, directed=directed)
    o.insert(s, d)
    o.insert(ns, nd)
    assert_same_adjacency(g, o)
    assert_sound(g)
    dead = np.unique(np.concatenate([rng.integers(0, n0, 30), rng.integers(n0, n, 30)])).astype(np.uint32)
    g.delete_vertices(dead)
    off, dst, _ = o.export()
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off).astype(np.int64))
    hit = np.isin(src, dead) | np.isin(dst, dead)
    o.delete(src[hit], dst[hit])
    assert_same_adjacency(g, o)
    assert_sound(g)
    x, sw = g.static_pagerank(0.85, 1e-6, 100)
    xo, _ = o.pagerank(0.85, 1e-6, 100, fixed_sweeps=sw)
    assert np.abs(x - xo).sum() < 1e-6
