"""GPU test of gv_pagerank_noalloc, the PageRank entry point that allocates
nothing (its scratch is a fixed device array inside libgv).  It exists for
callers that cannot allocate device memory at call time: serving threads
that must not stall on an allocation (cudaMalloc may synchronise the
device), and hosts whose device memory all belongs to their own arena.  The
test calls it through the C ABI and checks it against gv_pagerank, the
allocating entry point, on two calls in a row, and against the fp64 oracle.

This file is collected last on purpose; it must pass both alone in a fresh
process (the first call then sets up the device array's address) and after
the other tests."""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests.helpers import make_graph, rmat_graph

gv_b200 = pytest.importorskip("gv_b200")
pytestmark = pytest.mark.gpu

PR_L1 = 1e-6  # fp32 PageRank tolerance used across the suite


def _pagerank_device(lib, g, fn, n, torch, max_iter=100, eps=1e-6):
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    sweeps = C.c_int32()
    if fn == "noalloc":
        st = lib.gv_pagerank_noalloc(g.handle, 0.85, eps, max_iter, out.data_ptr(), C.byref(sweeps), None)
    else:
        st = lib.gv_pagerank(g.handle, 0.85, eps, max_iter, out.data_ptr(), C.byref(sweeps),
                             gv_b200.GV_MEM_DEVICE, None)
    assert st == 0, lib.gv_last_error_string().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64), sweeps.value


def _graph(scale, seed):
    n = 1 << scale
    s, d = rmat_graph(scale, 16, seed=seed)
    g = make_graph(n)
    g.batch_insert(s, d)
    g.synchronize()
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    return g, o, n


def test_noalloc_pagerank_matches_allocating_entry_point():
    import torch
    from gv_b200 import _lib
    lib = _lib.lib()
    g, o, n = _graph(12, 77)
    ref, ref_sweeps = _pagerank_device(lib, g, "alloc", n, torch)
    for call in range(2):  # two calls in a row share the device array
        x, sweeps = _pagerank_device(lib, g, "noalloc", n, torch)
        err = np.abs(x - ref).sum()
        xo, _ = o.pagerank(0.85, 1e-6, 100, fixed_sweeps=sweeps)
        err_o = np.abs(x - xo).sum()
        print(f"call {call}: sweeps {sweeps} vs {ref_sweeps}, L1 vs gv_pagerank {err:.3e}, vs fp64 {err_o:.3e}")
        assert abs(sweeps - ref_sweeps) <= 1
        assert err < PR_L1
        assert err_o < PR_L1
    g.close()


@pytest.mark.parametrize("max_iter", [5, 11])
def test_noalloc_stops_at_max_iter(max_iter):
    """epsilon 0 never converges, so the call ends on the sweep limit; an odd
    count leaves the result in the second iterate buffer."""
    import torch
    from gv_b200 import _lib
    lib = _lib.lib()
    g, o, n = _graph(11, 5)
    ref, ref_sweeps = _pagerank_device(lib, g, "alloc", n, torch, max_iter=max_iter, eps=0.0)
    xo, _ = o.pagerank(0.85, 0.0, max_iter, fixed_sweeps=max_iter)
    for _ in range(2):
        x, sweeps = _pagerank_device(lib, g, "noalloc", n, torch, max_iter=max_iter, eps=0.0)
        assert sweeps == max_iter == ref_sweeps
        assert np.abs(x - ref).sum() < PR_L1
        assert np.abs(x - xo).sum() < PR_L1
    g.close()


def test_noalloc_rejects_directed_store():
    import torch
    from gv_b200 import _lib
    lib = _lib.lib()
    g = make_graph(1024, directed=True)
    g.batch_insert(np.array([0, 1], np.uint32), np.array([1, 2], np.uint32))
    buf = torch.empty(1024, dtype=torch.float32, device="cuda")
    st = lib.gv_pagerank_noalloc(g.handle, 0.85, 1e-6, 10, buf.data_ptr(), None, None)
    assert st == _lib.GV_ERR_STATE
    g.close()


def test_noalloc_rejects_graphs_above_its_limit():
    from gv_b200 import _lib
    lib = _lib.lib()
    g = make_graph((1 << 20) + 1, pool_blocks=64)
    import torch
    buf = torch.empty(16, dtype=torch.float32, device="cuda")
    st = lib.gv_pagerank_noalloc(g.handle, 0.85, 1e-6, 10, buf.data_ptr(), None, None)
    assert st == _lib.GV_ERR_CAPACITY
    assert b"1048576" in lib.gv_last_error_string()
    g.close()
