"""GPU tests of ingest and snapshots: the device Matrix-Market parser returns
exactly the entries a line-by-line host parse finds (ids bit-exact, values
within one float ulp), a graph built from a file equals the oracle fed the
same pairs, and a snapshot loads back into the same store."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_same_adjacency, make_graph, rmat_graph, sample_existing

gv_b200 = pytest.importorskip("gv_b200")
pytestmark = pytest.mark.gpu


def _mtx_text(rng, n, k, values=True, last_newline=True):
    """Coordinate text with comments, blank lines, tabs, CRLF endings and
    several number formats; returns (text, src, dst, vals) 0-based."""
    s = rng.integers(1, n + 1, k)
    d = rng.integers(1, n + 1, k)
    v = rng.standard_normal(k) * 10.0 ** rng.integers(-4, 4, k)
    lines = ["%%MatrixMarket matrix coordinate " + ("real" if values else "pattern") + " general",
             "% generated", "", f"{n} {n} {k}"]
    for i in range(k):
        sep = "\t" if i % 7 == 0 else " "
        if values:
            fmt = ["{:.6g}", "{:.10e}", "{:.4f}", "{:d}"][i % 4]
            val = fmt.format(int(round(v[i] * 100)) if i % 4 == 3 else v[i])
            line = f"{s[i]}{sep}{d[i]}{sep}{val}"
        else:
            line = f"{s[i]}{sep}{d[i]}"
        if i % 5 == 0:
            line += "  "
        if i % 11 == 0:
            line += "\r"
        lines.append(line)
        if i % 97 == 0:
            lines.append("% interleaved comment")
    text = "\n".join(lines) + ("\n" if last_newline else "")
    vals = None
    if values:
        vals = np.array([float(l.split()[2]) for l in lines[4:] if l and not l.startswith("%")], np.float64)
    return text.encode(), (s - 1).astype(np.uint32), (d - 1).astype(np.uint32), vals


@pytest.mark.parametrize("on_device,last_newline", [(False, True), (True, False)])
def test_mtx_parse_matches_host_parse(on_device, last_newline):
    import torch
    rng = np.random.default_rng(3)
    text, s, d, v = _mtx_text(rng, 5000, 20000, values=True, last_newline=last_newline)
    arg = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda() if on_device else text
    meta, src, dst, val = gv_b200.mtx_parse(arg, with_values=True)
    if on_device:
        src, dst, val = (t.cpu().numpy() for t in (src, dst, val))
        src, dst = src.view(np.uint32), dst.view(np.uint32)
    assert meta["rows"] == 5000 and meta["entries"] == 20000 and not meta["pattern"]
    assert np.array_equal(src, s) and np.array_equal(dst, d)
    want = v.astype(np.float32)
    ulp = np.abs(want.view(np.int32).astype(np.int64) - val.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1


def test_mtx_parse_rejects_out_of_range_ids():
    text = b"%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\n4 1\n"
    with pytest.raises(gv_b200.GvError):
        gv_b200.mtx_parse(text)


@pytest.mark.parametrize("weighted", [False, True])
def test_graph_from_mtx_equals_oracle(tmp_path, weighted):
    rng = np.random.default_rng(7)
    n = 3000
    text, s, d, v = _mtx_text(rng, n, 15000, values=weighted)
    path = tmp_path / "g.mtx"
    path.write_bytes(text)
    g = gv_b200.GraphVine.from_mtx(path, weighted=weighted, directed=weighted, hbm_budget_bytes=1 << 30)
    assert g.n == n
    o = oracle.OracleGraph(n, directed=weighted, weighted=weighted)
    if weighted:
        o.insert(s, d, v.astype(np.float32))
    else:
        o.insert(s, d)
    assert_same_adjacency(g, o, weights=weighted)
    g.close()


@pytest.mark.parametrize("directed,weighted", [(False, False), (True, True)])
def test_snapshot_round_trip(tmp_path, directed, weighted):
    scale = 12
    n = 1 << scale
    s, d = rmat_graph(scale, 8, seed=9)
    rng = np.random.default_rng(9)
    w = rng.uniform(0.1, 1.0, len(s)).astype(np.float32) if weighted else None
    g = make_graph(n, directed=directed, weighted=weighted)
    g.batch_insert(s, d, w)
    off, dst, _ = g.export_csr()
    ds, dd = sample_existing(off, dst, 2000, rng)
    g.batch_delete(ds, dd)  # tombstones, no compaction
    g.synchronize()
    path = tmp_path / "g.snap"
    g.snapshot_save(path)
    h = gv_b200.GraphVine.snapshot_load(path, hbm_budget_bytes=1 << 30)
    assert h.n == n and h.directed == directed and h.weighted == weighted
    a_off, a_dst, a_w = g.export_csr(with_weights=weighted)
    b_off, b_dst, b_w = h.export_csr(with_weights=weighted)
    assert np.array_equal(a_off, b_off)
    src = np.repeat(np.arange(n, dtype=np.uint64), np.diff(a_off).astype(np.int64))
    ka = src * n + a_dst
    kb = src * n + b_dst
    oa, ob = np.argsort(ka), np.argsort(kb)
    assert np.array_equal(ka[oa], kb[ob])
    if weighted:
        assert np.array_equal(a_w[oa], b_w[ob])
    # one flipped byte in the payload is caught by the checksum
    raw = bytearray(path.read_bytes())
    raw[100] ^= 0x40
    path.write_bytes(bytes(raw))
    with pytest.raises(gv_b200.GvError):
        gv_b200.GraphVine.snapshot_load(path)
    g.close()
    h.close()
