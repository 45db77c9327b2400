"""The reference-API shim (include/graphvine.hpp): reference-style drivers
compile against libgv without a GPU (a plain C++ one with host containers,
and an nvcc one with thrust::device_vector results, as the reference's own
signatures take), and on a GPU they give the oracle's results (PageRank
within 1e-6 L1, exact triangle counts, BC within 1e-5), the batches of
CSR::generate_random_batch follow the reference's srand/rand draw sequence,
and the device accessors hold the last batch."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from tests.helpers import rmat_graph

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path("/usr/local/cuda")
LINK = ["-L", str(ROOT / "gv_b200"), "-lgv", f"-Wl,-rpath,{ROOT / 'gv_b200'}"]


def _build_host(tmp: Path) -> Path:
    exe = tmp / "compat_example"
    cmd = ["g++", "-O2", "-std=c++17", str(ROOT / "tests" / "compat_example.cpp"), "-I", str(ROOT / "include"),
           "-I", str(CUDA / "include"), *LINK, "-L", str(CUDA / "lib64"), "-lcudart",
           f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _build_thrust(tmp: Path) -> Path:
    exe = tmp / "compat_example_thrust"
    cmd = [str(CUDA / "bin" / "nvcc"), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           str(ROOT / "tests" / "compat_example_thrust.cu"), "-I", str(ROOT / "include"),
           "-Xlinker", f"-rpath,{ROOT / 'gv_b200'}", "-L", str(ROOT / "gv_b200"), "-lgv", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_host_shim_compiles_and_links(tmp_path):
    assert _build_host(tmp_path).exists()


def test_thrust_shim_compiles_and_links(tmp_path):
    assert _build_thrust(tmp_path).exists()


def _write_mtx(path: Path, n: int, s, d):
    pairs = {(min(a, b), max(a, b)) for a, b in zip(s.tolist(), d.tolist()) if a != b}
    with open(path, "w") as f:
        f.write(f"{n} {n} {len(pairs)}\n")
        for a, b in sorted(pairs):
            f.write(f"{a + 1} {b + 1}\n")
    return pairs


def reference_random_batch(n: int, batch_size: int, batch_number: int):
    """The draws of csr.cu:80-125 with this process's C library: per entry
    the source (rand() % n) and then the 1-based destination (rand() % n + 1),
    after srand(batch_number + 1).  Returns 0-based (src, dst)."""
    libc = ctypes.CDLL(None)
    libc.srand(batch_number + 1)
    s = np.empty(batch_size, np.uint32)
    d = np.empty(batch_size, np.uint32)
    for i in range(batch_size):
        s[i] = libc.rand() % n
        d[i] = libc.rand() % n
    return s, d


@pytest.mark.gpu
def test_reference_style_driver_matches_oracle(tmp_path):
    exe = _build_host(tmp_path)
    n = 1 << 10
    s, d = rmat_graph(10, 8, seed=12)
    _write_mtx(tmp_path / "g.mtx", n, s, d)
    rng = np.random.default_rng(1)
    ins_s, ins_d = rng.integers(0, n, 300), rng.integers(0, n, 300)
    _write_mtx(tmp_path / "i.mtx", n, ins_s, ins_d)
    del_s, del_d = s[:400], d[:400]
    _write_mtx(tmp_path / "d.mtx", n, del_s, del_d)
    out = subprocess.run([str(exe), str(tmp_path / "g.mtx"), str(tmp_path / "i.mtx"), str(tmp_path / "d.mtx"),
                          str(tmp_path / "res")], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    o.insert(ins_s.astype(np.uint32), ins_d.astype(np.uint32))
    o.delete(del_s, del_d)
    pr = np.fromfile(tmp_path / "res.pr", np.float32)
    tc = np.fromfile(tmp_path / "res.tc", np.float32)
    bc = np.fromfile(tmp_path / "res.bc", np.float32)
    opr, _ = o.pagerank(0.85, 1e-6, 100)
    assert np.abs(pr - opr).sum() < 1e-5  # oracle stops on its own sweep count here
    assert np.array_equal(tc.astype(np.uint64), o.tc()[0])
    ob = o.bc()
    nz = ob != 0
    assert np.max(np.abs(bc[nz] - ob[nz]) / ob[nz]) < 1e-5


@pytest.mark.gpu
def test_thrust_driver_matches_oracle_and_reference_batches(tmp_path):
    exe = _build_thrust(tmp_path)
    n = 1 << 11
    s, d = rmat_graph(11, 8, seed=44)
    _write_mtx(tmp_path / "g.mtx", n, s, d)
    bsz = 3000
    out = subprocess.run([str(exe), str(tmp_path / "g.mtx"), str(bsz), str(tmp_path / "r")],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "[BC] -> " in out.stdout
    # the batches follow the reference's draw sequence
    is_, id_ = reference_random_batch(n, bsz, 1)
    ds_, dd_ = reference_random_batch(n, bsz, 2)
    ins_off = np.fromfile(tmp_path / "r.ins_off", np.uint64)
    ins_edges = np.fromfile(tmp_path / "r.ins_edges", np.uint64)
    want_off = np.concatenate([[0], np.cumsum(np.bincount(is_, minlength=n))]).astype(np.uint64)
    assert np.array_equal(ins_off, want_off)
    for u in np.unique(is_)[:200]:  # per source, the destinations in draw order, 1-based
        a, b = int(ins_off[u]), int(ins_off[u + 1])
        assert np.array_equal(ins_edges[a:b], id_[is_ == u].astype(np.uint64) + 1)
    # affected flags after the insert batch: every endpoint of the graph's
    # entries (the constructor's bulk build) and of the batch (self-loops
    # are dropped before they mark anything)
    aff = np.fromfile(tmp_path / "r.affected", np.uint64)
    ends = np.zeros(n, bool)
    keep = s != d
    ends[s[keep]] = ends[d[keep]] = True
    keep_b = is_ != id_
    ends[is_[keep_b]] = ends[id_[keep_b]] = True
    assert np.array_equal(aff.astype(bool), ends)
    # the device accessors hold the delete batch
    del_off = np.fromfile(tmp_path / "r.del_off", np.uint64)
    del_edges = np.fromfile(tmp_path / "r.del_edges", np.uint64)
    del_deg = np.fromfile(tmp_path / "r.del_deg", np.uint64)
    assert np.array_equal(del_deg, np.bincount(ds_, minlength=n).astype(np.uint64))
    assert np.array_equal(np.diff(del_off), del_deg)
    assert np.array_equal(np.sort(del_edges), np.sort(dd_.astype(np.uint64) + 1))
    # results against the oracle: both batches applied symmetrically
    o = oracle.OracleGraph(n)
    o.insert(s, d)
    o.insert(is_, id_)
    o.delete(ds_, dd_)
    pr = np.fromfile(tmp_path / "r.pr", np.float32).astype(np.float64)
    pr_dyn = np.fromfile(tmp_path / "r.pr_dyn", np.float32).astype(np.float64)
    opr, osw = o.pagerank(0.85, 1e-6, 100)
    assert np.abs(pr - opr).sum() < 1e-5
    assert np.abs(pr_dyn - opr).sum() < 1e-5
    tc = np.fromfile(tmp_path / "r.tc", np.float32)
    tc_dyn = np.fromfile(tmp_path / "r.tc_dyn", np.float32)
    otc = o.tc()[0]
    assert np.array_equal(tc.astype(np.uint64), otc) and np.array_equal(tc_dyn.astype(np.uint64), otc)
