"""GPU tests of the request loop (gv_serve_trace): every query in a mixed
trace of updates and queries must return what the same query returns alone
on a graph holding the updates its epoch names (exactly those that arrived
before it, or at least those in the fresh mode), whether the loop runs
queries one at a time or several at once on views."""
import numpy as np
import pytest

import oracle
from tests.helpers import make_graph, rmat_graph, sample_existing

gv_b200 = pytest.importorskip("gv_b200")
pytestmark = pytest.mark.gpu

ALPHA, EPS = 0.85, 1e-6
PR_L1 = 1e-6
BC_REL = 1e-5


def _trace(n, s, d, rng, nreq=60, gap=0.0):
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    trace = []
    t = 0.0
    for i in range(nreq):
        r = rng.random()
        if r < 0.25:
            off, dst, _ = o.export()
            ins_s, ins_d = gv_b200.gen_uniform(n, int(rng.integers(20, 400)), seed=int(rng.integers(1 << 30)))
            del_s, del_d = sample_existing(off, dst, int(rng.integers(10, 200)), rng)
            o.insert(ins_s, ins_d)
            o.delete(del_s, del_d)
            trace.append(("update", ins_s, ins_d, del_s, del_d, t))
        elif r < 0.7:
            trace.append(("ppr", int(rng.integers(n)), t))
        elif r < 0.9:
            trace.append(("tc", rng.choice(n, int(rng.integers(1, 50)), replace=False).astype(np.uint32), t))
        else:
            trace.append(("bc", rng.choice(n, int(rng.integers(1, 5)), replace=False).astype(np.uint32), t))
        t += gap
    return trace


def _replay_and_check(n, s, d, trace, res, outs, fresh):
    """Applies the updates in trace order on a fresh graph (and the oracle)
    and runs each query alone after the updates its epoch says it saw: the
    first `epoch` update requests of the trace."""
    g = make_graph(n)
    g.batch_insert(s, d)
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    updates = [item for item in trace if item[0] == "update"]
    before = 0
    by_epoch = {}
    for i, item in enumerate(trace):
        assert res["status"][i] == 0, (i, res["status"][i])
        if item[0] == "update":
            before += 1
            continue
        # a query sees every update that arrived before it (exactly those unless fresh)
        if fresh:
            assert res["epoch"][i] >= before, (i, res["epoch"][i], before)
        else:
            assert res["epoch"][i] == before, (i, res["epoch"][i], before)
        by_epoch.setdefault(int(res["epoch"][i]), []).append(i)
    for e in range(len(updates) + 1):
        if e:
            item = updates[e - 1]
            g.batch_insert(item[1], item[2])
            g.batch_delete(item[3], item[4])
            g.compaction()
            o.insert(item[1], item[2])
            o.delete(item[3], item[4])
        for i in by_epoch.get(e, []):
            item = trace[i]
            if item[0] == "ppr":
                xo, _ = o.ppr(item[1], ALPHA, EPS, 100, fixed_sweeps=int(res["sweeps"][i]))
                assert np.abs(outs[i] - xo).sum() < PR_L1, i
            elif item[0] == "tc":
                assert np.array_equal(outs[i], g.tc_subset(item[1])), i
            else:
                ref = g.bc(item[1])
                assert np.allclose(outs[i], ref, rtol=BC_REL, atol=BC_REL), i
    g.close()


@pytest.mark.parametrize("slots,gap,fresh", [(1, 0.0, False), (4, 0.0, False), (4, 0.002, False),
                                             (4, 0.0, True), (4, 0.002, True)])
def test_mixed_trace_matches_each_query_alone(slots, gap, fresh):
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=21)
    trace = _trace(n, s, d, np.random.default_rng(5 + slots), gap=gap)
    g = make_graph(n)
    g.batch_insert(s, d)
    res, outs = g.serve(trace, slots=slots, ppr_batch=8, pace=gap > 0, alpha=ALPHA, epsilon=EPS, outputs=True,
                        fresh=fresh)
    g.synchronize()
    assert np.all(res["done_s"] >= res["start_s"])
    _replay_and_check(n, s, d, trace, res, outs, fresh)
    # the served graph ends equal to the replayed one
    g2 = make_graph(n)
    g2.batch_insert(s, d)
    for item in trace:
        if item[0] == "update":
            g2.batch_insert(item[1], item[2])
            g2.batch_delete(item[3], item[4])
    g2.compaction()
    a, b = g.export_csr(), g2.export_csr()
    assert np.array_equal(a[0], b[0])
    g.close()
    g2.close()


def test_fresh_mode_runs_arrived_queries_together():
    """Everything arrived at once: all updates go first and every query after
    the first update then runs on the last epoch, PPR queries in one launch."""
    scale = 11
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=6)
    trace = _trace(n, s, d, np.random.default_rng(17), nreq=40)
    nupd = sum(1 for t in trace if t[0] == "update")
    g = make_graph(n)
    g.batch_insert(s, d)
    res, _ = g.serve(trace, slots=4, ppr_batch=32, pace=False, fresh=True)
    q = [i for i, t in enumerate(trace) if t[0] != "update"]
    first_u = min(i for i, t in enumerate(trace) if t[0] == "update")
    for i in q:
        assert res["epoch"][i] == (0 if i < first_u else nupd), i
    ppr_groups = {int(res["group"][i]) for i in q if trace[i][0] == "ppr" and i > first_u}
    assert len(ppr_groups) == 1
    g.close()


def test_budget_of_one_byte_runs_groups_one_at_a_time():
    scale = 11
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=4)
    rng = np.random.default_rng(9)
    trace = [("ppr", int(v), 0.0) for v in rng.choice(n, 10, replace=False)]
    trace += [("tc", rng.choice(n, 5, replace=False).astype(np.uint32), 0.0)]
    trace += [("bc", np.array([1, 2], np.uint32), 0.0)]
    g = make_graph(n)
    g.batch_insert(s, d)
    res, _ = g.serve(trace, slots=4, ppr_batch=4, pace=False, hbm_budget_bytes=1)
    spans = sorted({(int(r["group"]), float(r["start_s"]), float(r["done_s"])) for r in res})
    assert len(spans) == 5  # 3 PPR groups of <= 4, one TC group, one BC
    spans.sort(key=lambda t: t[1])
    for a, b in zip(spans, spans[1:]):
        assert b[1] >= a[2], (a, b)
    g.close()


def test_bc_queries_run_in_pairs():
    scale = 11
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=12)
    rng = np.random.default_rng(31)
    trace = [("bc", rng.choice(n, k, replace=False).astype(np.uint32), 0.0) for k in (3, 32, 20)]
    g = make_graph(n)
    g.batch_insert(s, d)
    res, outs = g.serve(trace, slots=2, pace=False, outputs=True)
    assert res["group"][0] == res["group"][1] != res["group"][2]
    for i, item in enumerate(trace):
        assert np.allclose(outs[i], g.bc(item[1]), rtol=BC_REL, atol=BC_REL), i
    g.close()


def test_serve_rejects_bad_config_and_views():
    n = 256
    g = make_graph(n)
    with pytest.raises(gv_b200.GvError):
        g.serve([("ppr", 0, 0.0)], ppr_batch=33)
    v = g.view()
    with pytest.raises(gv_b200.GvError):
        v.serve([("ppr", 0, 0.0)])
    with pytest.raises(gv_b200.GvError):
        v.batch_insert(np.array([1], np.uint32), np.array([2], np.uint32))
    v.close()
    g.close()
