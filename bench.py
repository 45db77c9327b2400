#!/usr/bin/env python3
"""Benchmark of the GraphVine dynamic-graph hot path on B200.

Workload (one step = one update batch of the plain method at scale):
  undirected R-MAT scale 22, edge factor 16, a/b/c/d = 0.57/0.19/0.19/0.05,
  seeded; each step applies 1M updates (500K inserts of uniform-random new
  pairs + 500K deletes of existing edges), compacts, then runs PageRank
  (fp32, alpha 0.85, L1 1e-6, <= 100 sweeps) and an exact triangle count;
  every 5th step also runs betweenness centrality from 64 seeded sources.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gv|reference]

Prints one JSON line (rank 0).  `value` = edge updates/s over the timed
steps with the batches already resident in HBM; `e2e` = the same through the
C-ABI with pinned host buffers, copies inside the timed region.  For N > 1
every rank runs an independent replica (the path does not shard).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "edge updates/s & PageRank GTEPS, plain vs batched/served, % of HBM peak"
ALPHA, EPS, MAX_ITER = 0.85, 1e-6, 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gv", "reference"], default="gv")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--batch", type=int, default=1_000_000, help="updates per step (half inserts, half deletes)")
    ap.add_argument("--bc-every", type=int, default=5)
    ap.add_argument("--bc-sources", type=int, default=64)
    ap.add_argument("--block", type=int, default=128)
    ap.add_argument("--tpv", type=int, default=16)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-batching", action="store_true", help="skip the scale-24 batched-vs-plain section")
    ap.add_argument("--batch-scale", type=int, default=24)
    ap.add_argument("--c3-batches", type=int, default=64)
    ap.add_argument("--no-incremental", action="store_true", help="skip the incremental triangle-count section")
    ap.add_argument("--no-ingest", action="store_true", help="skip the Matrix-Market / snapshot section")
    ap.add_argument("--ingest-scale", type=int, default=20)
    ap.add_argument("--no-diff", action="store_true", help="skip the scale-20 differentiation section")
    ap.add_argument("--diff-scale", type=int, default=20)
    ap.add_argument("--fd-edges", type=int, default=64)
    ap.add_argument("--no-serving", action="store_true", help="skip the scale-25 serving section")
    ap.add_argument("--serve-scale", type=int, default=25)
    ap.add_argument("--serve-requests", type=int, default=120)
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--serve-load", type=float, default=0.7, help="Poisson rate as a fraction of served capacity")
    ap.add_argument("--serve-hbm", type=int, default=96, help="GB of HBM the serving loop may give queries")
    return ap.parse_args()


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        """Starts nvidia-smi and waits for its first sample, so its start-up
        (NVML initialisation) is over before the timed region begins."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        t_wait = time.monotonic() + 10.0
        while not self.lines and time.monotonic() < t_wait:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self, t0: float | None = None, t1: float | None = None) -> dict | None:
        """Summary of the samples taken in [t0, t1] (host monotonic time; all
        samples when no window is given or none falls inside it)."""
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = [ln for t, ln in self.lines if t0 is not None and t0 <= t <= t1 + 0.2]
        for ln in inside or [ln for _, ln in self.lines]:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


# ------------------------------------------------------------------- workload
def make_batches(n, off, dst, steps, half, seed):
    """Per step: uniform new pairs to insert, existing undirected edges to delete."""
    import gv_b200
    deg = np.diff(off).astype(np.int64)
    src_of = np.repeat(np.arange(n, dtype=np.uint32), deg)
    und = np.nonzero(src_of < dst)[0]  # each undirected edge once
    rng = np.random.default_rng(seed)
    picks = rng.choice(len(und), size=min(len(und), steps * half), replace=False)
    out = []
    for b in range(steps):
        ins_s, ins_d = gv_b200.gen_uniform(n, half, seed=seed * 1000 + b)
        sel = und[picks[b * half:(b + 1) * half]]
        out.append((ins_s, ins_d, src_of[sel].copy(), dst[sel].copy()))
    return out


def bc_sources(n, k, seed):
    return np.random.default_rng(seed + 7).choice(n, size=k, replace=False).astype(np.uint32)


def zipf_ids(rng, n, k, a=1.1):
    """k vertex ids, Zipf(a)-skewed over a seeded permutation of [0, n)."""
    out = np.empty(0, np.int64)
    while len(out) < k:
        z = rng.zipf(a, size=2 * (k - len(out)))
        out = np.concatenate([out, z[z <= n] - 1])
    out = out[:k]
    mult = 0x9E3779B1 | 1  # odd multiplier: a bijection on [0, 2^scale)
    return ((out * mult + 12345) & (n - 1)).astype(np.uint32)


def make_c3_batches(n, off, dst, nb, seed, lo=1_000, hi=4_000_000):
    """nb batches: sizes log-uniform in [lo, hi], insert fraction U[0.2, 0.8],
    sources Zipf(1.1); inserts pair a source with a uniform vertex, deletes
    pick an existing neighbour of the source."""
    rng = np.random.default_rng(seed)
    deg = np.diff(off).astype(np.int64)
    batches = []
    for _ in range(nb):
        size = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        ni = int(size * rng.uniform(0.2, 0.8))
        nd = size - ni
        ins_s = zipf_ids(rng, n, ni)
        ins_d = rng.integers(0, n, ni, dtype=np.int64).astype(np.uint32)
        cand = zipf_ids(rng, n, 2 * nd + 16)
        cand = cand[deg[cand] > 0][:nd]
        pick = (rng.random(len(cand)) * deg[cand]).astype(np.int64)
        del_s = cand
        del_d = dst[off[cand].astype(np.int64) + pick]
        batches.append((ins_s, ins_d, del_s.astype(np.uint32), del_d.astype(np.uint32)))
    return batches


# ----------------------------------------------------------------- CPU legs
def cpu_sample(args, pairs, batches, n, threads, steps):
    """Times the oracle (the reference's semantics restated on the CPU) on
    `steps` steps of the same workload; BC is timed on 4 sources and scaled."""
    import oracle
    oracle.set_threads(threads)
    g = oracle.OracleGraph(n)
    g.insert(*pairs)
    src = bc_sources(n, args.bc_sources, args.seed)
    times = []
    detail = {}
    for b in range(steps):
        ins_s, ins_d, del_s, del_d = batches[b % len(batches)]
        t0 = time.perf_counter()
        g.insert(ins_s, ins_d)
        g.delete(del_s, del_d)
        t1 = time.perf_counter()
        g.pagerank(ALPHA, EPS, MAX_ITER)
        t2 = time.perf_counter()
        g.tc()
        t3 = time.perf_counter()
        g.bc(src[:4])
        t4 = time.perf_counter()
        bc_amortised = (t4 - t3) * (args.bc_sources / 4) / args.bc_every
        times.append((t3 - t0) + bc_amortised)
        detail = {"update_s": t1 - t0, "pagerank_s": t2 - t1, "tc_s": t3 - t2, "bc_4src_s": t4 - t3}
    return sum(times) / len(times), detail


def run_reference(args, rank, world):
    if rank != 0:
        return
    import gv_b200
    n = 1 << args.scale
    pairs = gv_b200.gen_rmat(args.scale, args.edge_factor << args.scale, args.seed)
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    g = oracle.OracleGraph(n)
    g.insert(*pairs)
    off, dst, _ = g.export()
    half = args.batch // 2
    batches = make_batches(n, off, dst, args.warmup + args.steps, half, args.seed)
    del g
    step_s, detail = cpu_sample(args, pairs, batches, n, threads, args.warmup + args.steps)
    value = args.batch / step_s
    sample = (f"oracle port (C++/OpenMP, {threads} threads): {args.warmup + args.steps} full steps of the "
              f"workload (insert+delete+PageRank+TC); BC timed on 4 of {args.bc_sources} sources, scaled "
              f"and amortised over {args.bc_every} steps")
    line = {"metric": METRIC, "value": value, "unit": "edge updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded R-MAT, uniform inserts, sampled deletes)",
            "impl": "reference",
            "config": workload_config(args, n, int(off[-1])),
            "cpu_baseline": {"value": value, "unit": "edge updates/s", "cores": threads, "kind": "port",
                             "sample": sample, "phases_s": detail},
            "e2e": {"value": value, "unit": "edge updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def max_over_ranks(values, device, dist=None):
    """Element-wise maximum of each rank's timings (every rank gets it): the
    job is as slow as its slowest replica."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def workload_config(args, n, m0):
    return {"workload": (f"plain method at scale: undirected R-MAT scale {args.scale} ef {args.edge_factor}; "
                         f"per step {args.batch} updates ({args.batch // 2} inserts + {args.batch // 2} deletes) "
                         f"+ compaction + PageRank + exact TC; BC from {args.bc_sources} sources every "
                         f"{args.bc_every} steps"),
            "scale": args.scale, "n": n, "m_initial_entries": m0, "batch_updates": args.batch,
            "block_size": args.block, "threads_per_vertex": args.tpv,
            "l2": "working set larger than L2 (adjacency ~0.5 GB vs 126 MB); each step uses fresh batch buffers",
            "parallelism": "replicas"}


# ------------------------------------------------------------ batching leg
def insert_chunked(g, s_dev, d_dev, chunk=1 << 26):
    for i in range(0, len(s_dev), chunk):
        g.batch_insert(s_dev[i:i + chunk], d_dev[i:i + chunk])
    g.synchronize()


def run_batching(args, dev):
    """Batching workload: 64 uneven Zipf batches on R-MAT scale 24, plain
    (one synchronous call per batch + compaction, as the reference) against
    the batched window; 32 PPR queries one by one against one batched call."""
    import torch
    import gv_b200
    scale = args.batch_scale
    n = 1 << scale
    seed = args.seed + 100
    # autotune on a scale-20 sample of the same workload shape
    ts, td = gv_b200.gen_rmat(20, 16 << 20, seed)
    to = gv_b200.GraphVine(1 << 20, hbm_budget_bytes=4 << 30)
    to.batch_insert(ts, td)
    toff, tdst, _ = to.export_csr()
    to.close()
    tune_batches = make_c3_batches(1 << 20, toff, tdst, 16, seed, hi=200_000)
    best, tune = gv_b200.autotune(1 << 20, ts, td, tune_batches, hbm_budget_bytes=4 << 30)
    cfg = dict(block_size=best["block_size"], threads_per_vertex=best["threads_per_vertex"],
               hbm_budget_bytes=24 << 30, max_batch_pairs=1 << 22, device=dev.index or 0)
    s_dev, d_dev = gv_b200.gen_rmat(scale, args.edge_factor << scale, seed, device=dev)
    gp = gv_b200.GraphVine(n, **cfg)
    insert_chunked(gp, s_dev, d_dev)
    off, dst, _ = gp.export_csr()
    m0 = int(off[-1])
    batches = make_c3_batches(n, off, dst, args.c3_batches, seed)
    del off, dst
    gb = gv_b200.GraphVine(n, **cfg)
    insert_chunked(gb, s_dev, d_dev)
    del s_dev, d_dev
    torch.cuda.empty_cache()
    tot = sum(len(b[0]) + len(b[2]) for b in batches)
    dev_b = [tuple(torch.from_numpy(a.view(np.int32)).to(dev) for a in b) for b in batches]
    descs, srcs, dsts, p = [], [], [], 0
    for a, b_, c, e in batches:
        descs.append((p, len(a), len(c)))
        srcs += [a, c]
        dsts += [b_, e]
        p += len(a) + len(c)
    wsrc = torch.from_numpy(np.concatenate(srcs).view(np.int32)).to(dev)
    wdst = torch.from_numpy(np.concatenate(dsts).view(np.int32)).to(dev)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    for ins_s, ins_d, del_s, del_d in dev_b:
        gp.batch_insert(ins_s, ins_d)
        gp.synchronize()
        gp.batch_delete(del_s, del_d)
        gp.synchronize()
        gp.compaction()
        gp.synchronize()
    e[1].record()
    torch.cuda.synchronize()
    e[2].record()
    gb.batch_run((descs, wsrc, wdst), compact=True, graph=True)
    gb.synchronize()
    e[3].record()
    torch.cuda.synchronize()
    plain_ms, batched_ms = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
    m_p, m_b = gp.num_edges(), gb.num_edges()
    # PageRank queries: 32 sources one by one vs one batched call
    srcs_q = np.random.default_rng(seed).choice(n, 32, replace=False).astype(np.uint32)
    xq = torch.empty(n, dtype=torch.float32, device=dev)
    xb = torch.empty((n, 32), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    e[0].record()
    sw_plain = 0
    for sq in srcs_q:
        _, sw = gp.ppr(int(sq), out=xq)
        sw_plain += sw
    e[1].record()
    torch.cuda.synchronize()
    e[2].record()
    _, sw_b = gb.ppr_batch(srcs_q, out=xb)
    e[3].record()
    torch.cuda.synchronize()
    pr_plain_ms, pr_batched_ms = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
    gteps_plain = m_p * sw_plain / (pr_plain_ms / 1e3) / 1e9
    gteps_batched = m_b * sw_b * 32 / (pr_batched_ms / 1e3) / 1e9
    gp.close()
    gb.close()
    return {"workload": (f"R-MAT scale {scale} ef {args.edge_factor}, {len(batches)} batches log-uniform in "
                         f"[1K, 4M] updates, Zipf(1.1) sources, insert fraction U[0.2, 0.8]; 32 PPR queries"),
            "m_initial_entries": m0, "updates": tot, "edges_after_plain": m_p, "edges_after_batched": m_b,
            "plain_updates_per_s": tot / (plain_ms / 1e3), "batched_updates_per_s": tot / (batched_ms / 1e3),
            "updates_speedup": plain_ms / batched_ms,
            "plain": "one synchronous insert, delete and compaction call per batch",
            "batched": "gv_batch_run: one coalesced window, compaction once, CUDA graph",
            "pagerank_gteps_plain": gteps_plain, "pagerank_gteps_batched": gteps_batched,
            "pagerank_speedup": pr_plain_ms / pr_batched_ms,
            "autotune_best": best, "autotune": tune}


def run_differentiation(args):
    """Differentiation workload: directed weighted R-MAT (weights uniform in
    (0.1, 1], normalised per row), weighted PageRank forward, then the
    gradient of sum(c_i x_i), c ~ N(0, 1), with respect to every raw edge
    weight through the adjoint solve; the gradient of args.fd_edges random
    edges is checked against fp64 central differences (h = 1e-6) of the
    oracle on the host."""
    import torch
    import gv_b200
    import oracle
    scale = args.diff_scale
    n = 1 << scale
    seed = args.seed + 300
    rng = np.random.default_rng(seed)
    s, d = gv_b200.gen_rmat(scale, args.edge_factor << scale, seed)
    w = (1.0 - 0.9 * rng.random(len(s))).astype(np.float32)
    c = rng.standard_normal(n)
    g = gv_b200.GraphVine(n, directed=True, weighted=True, hbm_budget_bytes=8 << 30, max_batch_pairs=len(s))
    g.batch_insert(s, d, w)
    g.synchronize()
    m = g.num_edges()
    tol, it = 1e-7, 200
    g.wpr_forward(ALPHA, tol, it)  # warm-up (scratch)
    c32 = c.astype(np.float32)
    torch.cuda.synchronize()
    gv_b200.profile_reset()
    gv_b200.profile_enable(True)
    t0 = time.perf_counter()
    x, sw_f = g.wpr_forward(ALPHA, tol, it)
    torch.cuda.synchronize()
    fwd_s = time.perf_counter() - t0
    g.wpr_backward(x, c32, ALPHA, tol, it, mode=0)  # warm-up
    torch.cuda.synchronize()
    prof_f = {k: gv_b200.profile_query(k) for k in ("wpr_build", "wpr_sweep")}
    gv_b200.profile_reset()
    t0 = time.perf_counter()
    grad, lam, sw_b = g.wpr_backward(x, c32, ALPHA, tol, it, mode=0)
    torch.cuda.synchronize()
    bwd_s = time.perf_counter() - t0
    prof_b = {k: gv_b200.profile_query(k) for k in ("pull", "wpr_grad")}
    gv_b200.profile_enable(False)
    off, dst, _ = g.export_csr()
    g.close()
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off).astype(np.int64))
    ks = rng.choice(len(dst), args.fd_edges, replace=False)
    o = oracle.OracleGraph(n, directed=True, weighted=True)
    o.insert(s, d, w)
    t0 = time.perf_counter()
    fd = o.wpr_fd(c, src[ks], dst[ks], 1e-6)
    fd_s = time.perf_counter() - t0
    del o
    err = np.abs(grad[ks].astype(np.float64) - fd)
    scale_fd = float(np.abs(fd).max())
    return {"workload": (f"directed R-MAT scale {scale} ef {args.edge_factor}, weights U(0.1, 1] normalised per row; "
                         f"weighted PageRank (alpha {ALPHA}, L1 tol {tol}) and d(sum c_i x_i)/d(raw weight) for "
                         f"every entry, c ~ N(0, 1)"),
            "m_entries": m, "forward_ms": fwd_s * 1e3, "forward_sweeps": sw_f,
            "forward_gteps": m * sw_f / fwd_s / 1e9,
            "forward_device_ms": {"transpose_build": prof_f["wpr_build"][0], "sweeps": prof_f["wpr_sweep"][0]},
            "forward_sweep_gteps": m * sw_f / (prof_f["wpr_sweep"][0] / 1e3) / 1e9 if prof_f["wpr_sweep"][0] else None,
            "backward_ms": bwd_s * 1e3, "adjoint_sweeps": sw_b,
            "backward_device_ms": {"adjoint_sweeps": prof_b["pull"][0], "gradient": prof_b["wpr_grad"][0]},
            "adjoint_sweep_gteps": m * sw_b / (prof_b["pull"][0] / 1e3) / 1e9 if prof_b["pull"][0] else None,
            "backward_note": "adjoint solve + one gradient entry per stored entry, returned to the host in export order",
            "fd_check": {"edges": int(args.fd_edges), "h": 1e-6, "kind": "fp64 central differences (oracle, host)",
                         "max_abs_err": float(err.max()), "max_abs_fd": scale_fd,
                         "max_err_over_max_fd": float(err.max() / scale_fd) if scale_fd else None,
                         "oracle_seconds": fd_s}}


def run_ingest(args):
    """Ingest workload: R-MAT scale args.ingest_scale written as Matrix-Market
    text (1-based \"src dst\" lines), parsed on the device from host memory
    (copy included) and from device memory; then a snapshot of the built graph
    saved and loaded back."""
    import tempfile
    import torch
    import gv_b200
    scale = args.ingest_scale
    n = 1 << scale
    s, d = gv_b200.gen_rmat(scale, args.edge_factor << scale, args.seed + 400)
    # fixed-width, zero-padded ids (valid decimal), built as a byte matrix
    width = len(str(n))
    rows = np.empty((len(s), 2 * width + 2), np.uint8)
    for col, ids in ((0, s.astype(np.int64) + 1), (width + 1, d.astype(np.int64) + 1)):
        for j in range(width):
            rows[:, col + width - 1 - j] = ord("0") + (ids // 10 ** j) % 10
    rows[:, width] = ord(" ")
    rows[:, -1] = ord("\n")
    text = f"%%MatrixMarket matrix coordinate pattern general\n{n} {n} {len(s)}\n".encode() + rows.tobytes()
    del rows
    host = torch.frombuffer(bytearray(text), dtype=torch.uint8).pin_memory()
    dev = host.cuda()
    gv_b200.mtx_parse(dev)  # warm-up
    # each call sizes and parses the text and allocates its own scratch and
    # outputs, whose allocation time varies from call to call: best of five
    times = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        meta, src, dst, _ = gv_b200.mtx_parse(dev)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    dev_s = min(times)
    ok = bool(np.array_equal(src[:1000].cpu().numpy().view(np.uint32), s[:1000]))
    t0 = time.perf_counter()
    gv_b200.mtx_parse(host.numpy().tobytes())
    host_s = time.perf_counter() - t0
    out = {"workload": f"R-MAT scale {scale} ef {args.edge_factor} as Matrix-Market text",
           "text_bytes": len(text), "entries": int(meta["entries"]), "first_entries_match": ok,
           "device_text_gb_s": len(text) / dev_s / 1e9, "device_text_entries_per_s": meta["entries"] / dev_s,
           "device_calls_s": times,
           "host_text_gb_s": len(text) / host_s / 1e9,
           "host_note": "host text: pageable copy, host header read, device parse and copy back of the ids"}
    with tempfile.TemporaryDirectory() as td:
        g = gv_b200.GraphVine(n, max_batch_pairs=len(s))
        g.batch_insert(s, d)
        g.synchronize()
        path = f"{td}/g.snap"
        t0 = time.perf_counter()
        g.snapshot_save(path)
        save_s = time.perf_counter() - t0
        m = g.num_edges()
        g.close()
        t0 = time.perf_counter()
        h = gv_b200.GraphVine.snapshot_load(path)
        load_s = time.perf_counter() - t0
        same = h.num_edges() == m
        h.close()
    out.update({"snapshot_entries": m, "snapshot_save_s": save_s, "snapshot_load_s": load_s, "snapshot_same_m": same})
    return out


def make_serve_trace(n, s_dev, d_dev, nreq, seed):
    """Serving requests: 60% update batches (log-uniform 1K-1M updates, half
    inserts of uniform-random pairs, half deletes sampled from the graph's
    generated pairs), 40% queries split evenly between PPR from a random
    source, incident triangles of 10K random vertices and BC from 32 sampled
    sources.  Arrival times are set by the caller."""
    import torch
    import gv_b200
    rng = np.random.default_rng(seed)
    items = []
    m = len(s_dev)
    for _ in range(nreq):
        r = rng.random()
        if r < 0.6:
            k = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
            ni = k // 2
            ins_s, ins_d = gv_b200.gen_uniform(n, ni, seed=int(rng.integers(1 << 62)))
            idx = torch.from_numpy(rng.integers(0, m, k - ni)).to(s_dev.device)
            del_s = s_dev[idx].cpu().numpy().view(np.uint32)
            del_d = d_dev[idx].cpu().numpy().view(np.uint32)
            items.append(("update", ins_s, ins_d, del_s, del_d))
        elif r < 0.6 + 0.4 / 3:
            items.append(("ppr", int(rng.integers(n))))
        elif r < 0.6 + 0.8 / 3:
            v = np.unique(rng.integers(0, n, 10_200))[:10_000]
            items.append(("tc", rng.permutation(v).astype(np.uint32)))
        else:
            items.append(("bc", np.unique(rng.integers(0, n, 40))[:32].astype(np.uint32)))
    return items


def _pct(a, q):
    return float(np.percentile(np.asarray(a), q)) if len(a) else None


def run_serving(args, dev):
    """Serving workload: a resident R-MAT scale-25 graph and a seeded request
    trace.  plain = every request through its own synchronous call in trace
    order; served = gv_serve_trace with everything arrived (throughput); paced
    = gv_serve_trace with Poisson arrivals at a fraction of the served
    capacity (p50 / p99 latency)."""
    import torch
    import gv_b200
    scale = args.serve_scale
    n = 1 << scale
    seed = args.seed + 200
    cfg = dict(block_size=args.block, threads_per_vertex=args.tpv, hbm_budget_bytes=48 << 30,
               max_batch_pairs=1 << 22, device=dev.index or 0)
    s_dev, d_dev = gv_b200.gen_rmat(scale, args.edge_factor << scale, seed, device=dev)
    items = make_serve_trace(n, s_dev, d_dev, args.serve_requests, seed)
    kinds = [it[0] for it in items]
    upd_pairs = sum(len(it[1]) + len(it[3]) for it in items if it[0] == "update")

    def build():
        g = gv_b200.GraphVine(n, **cfg)
        insert_chunked(g, s_dev, d_dev)
        g.compaction()
        g.synchronize()
        return g

    # plain: one synchronous call per request, results left on the device
    g = build()
    m0 = g.num_edges()
    xq = torch.empty(n, dtype=torch.float32, device=dev)
    bq = torch.empty(n, dtype=torch.float32, device=dev)
    lib = gv_b200._lib.lib()
    t_kind = {"update": 0.0, "ppr": 0.0, "tc": 0.0, "bc": 0.0}
    ppr_edges = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in items:
        ta = time.perf_counter()
        if it[0] == "update":
            g.batch_insert(it[1], it[2])
            g.batch_delete(it[3], it[4])
            g.compaction()
            g.synchronize()
        elif it[0] == "ppr":
            _, sw = g.ppr(it[1], ALPHA, EPS, MAX_ITER, out=xq)
            ppr_edges += m0 * sw
        elif it[0] == "tc":
            g.tc_subset(it[1])
        else:
            src = torch.from_numpy(np.ascontiguousarray(it[1], np.uint32).view(np.int32)).to(dev)
            gv_b200._check(lib.gv_bc(g._h, src.data_ptr(), len(src), bq.data_ptr(), gv_b200.GV_MEM_DEVICE, 0),
                           "gv_bc")
            torch.cuda.synchronize()
        t_kind[it[0]] += time.perf_counter() - ta
    plain_s = time.perf_counter() - t0
    g.close()

    # served, everything arrived at t = 0
    def trace(arrivals):
        return [it + (float(a),) for it, a in zip(items, arrivals)]

    g = build()
    t0 = time.perf_counter()
    res, _ = g.serve(trace(np.zeros(len(items))), slots=args.serve_slots, ppr_batch=32, pace=False,
                     alpha=ALPHA, epsilon=EPS, max_iter=MAX_ITER, hbm_budget_bytes=args.serve_hbm << 30)
    served_s = time.perf_counter() - t0
    g.close()
    assert np.all(res["status"] == 0)

    def group_time(res, kind):
        spans = {}
        for i, k in enumerate(kinds):
            if k == kind:
                spans[int(res["group"][i])] = float(res["done_s"][i] - res["start_s"][i])
        return sum(spans.values())

    ppr_edges_served = sum(m0 * int(res["sweeps"][i]) for i, k in enumerate(kinds) if k == "ppr")
    served = {"makespan_s": served_s, "requests_per_s": len(items) / served_s,
              "updates_per_s": upd_pairs / served_s,
              "update_engine_updates_per_s": upd_pairs / max(group_time(res, "update"), 1e-9),
              "ppr_gteps": ppr_edges_served / max(group_time(res, "ppr"), 1e-9) / 1e9,
              "groups": int(len(np.unique(res["group"])))}
    plain = {"makespan_s": plain_s, "requests_per_s": len(items) / plain_s, "updates_per_s": upd_pairs / plain_s,
             "update_engine_updates_per_s": upd_pairs / max(t_kind["update"], 1e-9),
             "ppr_gteps": ppr_edges / max(t_kind["ppr"], 1e-9) / 1e9,
             "seconds_by_kind": t_kind}

    # paced: Poisson arrivals at a fraction of the served capacity
    rate = args.serve_load * len(items) / served_s
    arr = np.cumsum(np.random.default_rng(seed + 1).exponential(1.0 / rate, len(items)))
    arr -= arr[0]
    g = build()
    res, _ = g.serve(trace(arr), slots=args.serve_slots, ppr_batch=32, pace=True, alpha=ALPHA, epsilon=EPS,
                     max_iter=MAX_ITER, hbm_budget_bytes=args.serve_hbm << 30)
    g.close()
    del s_dev, d_dev
    torch.cuda.empty_cache()
    lat = res["latency_ms"]
    span = float(res["done_s"].max() - arr[0])
    per_kind = {}
    for k in ("update", "ppr", "tc", "bc"):
        sel = [lat[i] for i in range(len(items)) if kinds[i] == k]
        per_kind[k] = {"count": len(sel), "p50_ms": _pct(sel, 50), "p99_ms": _pct(sel, 99)}
    return {"workload": (f"R-MAT scale {scale} ef {args.edge_factor} resident; {len(items)} requests: 60% update "
                         f"batches (log-uniform 1K-1M updates, 50/50), 40% queries (PPR / TC over 10K vertices / "
                         f"BC from 32 sources)"),
            "m_initial_entries": m0, "update_pairs": upd_pairs,
            "mix": {k: kinds.count(k) for k in ("update", "ppr", "tc", "bc")},
            "plain": plain, "served": served,
            "served_vs_plain": {"requests": plain_s / served_s,
                                "updates_per_s": served["updates_per_s"] / plain["updates_per_s"],
                                "ppr_gteps": served["ppr_gteps"] / plain["ppr_gteps"] if plain["ppr_gteps"] else None},
            "paced": {"poisson_rate_per_s": rate, "load": args.serve_load, "slots": args.serve_slots,
                      "hbm_budget_gb": args.serve_hbm, "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99),
                      "throughput_requests_per_s": len(items) / span, "updates_per_s": upd_pairs / span,
                      "by_kind": per_kind}}


# ------------------------------------------------------------------ GPU leg
def run_gv(args, rank, world, local_rank):
    import torch
    import gv_b200
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = 1 << args.scale
    seed = args.seed + rank
    g = gv_b200.GraphVine(n, block_size=args.block, threads_per_vertex=args.tpv, device=local_rank,
                          max_batch_pairs=args.batch)
    s_dev, d_dev = gv_b200.gen_rmat(args.scale, args.edge_factor << args.scale, seed, device=dev)
    g.batch_insert(s_dev, d_dev)
    g.synchronize()
    del s_dev, d_dev
    torch.cuda.empty_cache()
    off, dst, _ = g.export_csr()
    m0 = int(off[-1])
    half = args.batch // 2
    total_steps = args.warmup + args.steps + (0 if args.no_e2e else args.steps)
    n_incr = 0 if (args.no_incremental or world > 1) else 4
    batches = make_batches(n, off, dst, total_steps + 2 * n_incr + (1 if n_incr else 0), half, seed)
    srcs = bc_sources(n, args.bc_sources, seed)
    dev_batches = [tuple(torch.from_numpy(a.astype(np.int32)).to(dev) for a in b) for b in batches]
    x_dev = torch.empty(n, dtype=torch.float32, device=dev)
    bc_dev = torch.empty(n, dtype=torch.float32, device=dev)
    src_dev = torch.from_numpy(srcs.astype(np.int32)).to(dev)

    stats = {"pr_sweeps": [], "m": [], "tc_work": [], "triangles": []}

    def step(b, inputs, host_out=None):
        ins_s, ins_d, del_s, del_d = inputs
        g.batch_insert(ins_s, ins_d)
        g.batch_delete(del_s, del_d)
        g.compaction()
        if host_out is None:
            _, sw = g.static_pagerank(ALPHA, EPS, MAX_ITER, out=x_dev)
        else:
            _, sw = g.static_pagerank(ALPHA, EPS, MAX_ITER, out=host_out["x"])
        _, tri = g.static_tc(per_vertex=False)
        stats["pr_sweeps"].append(sw)
        stats["triangles"].append(tri)
        if (b % args.bc_every) == args.bc_every - 1:
            if host_out is None:
                lib = gv_b200._lib.lib()
                gv_b200._check(lib.gv_bc(g._h, src_dev.data_ptr(), len(srcs), bc_dev.data_ptr(),
                                         gv_b200.GV_MEM_DEVICE, 0), "gv_bc")
            else:
                host_out["bc"][:] = g.bc(srcs)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    if not args.no_clocks:
        sampler.start()
    # warm-up; a BC call as well when no warm-up step ran one, so the BC
    # scratch is sized before the timed region like everything else
    for b in range(args.warmup):
        step(b, dev_batches[b])
    if args.warmup < args.bc_every:
        g.bc(srcs)
    barrier()
    for k in stats:
        stats[k].clear()
    gv_b200.profile_reset()
    gv_b200.profile_enable(True)
    launches0 = gv_b200.kernel_launches()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    barrier()
    h_start = time.monotonic()
    t_start.record()
    for i in range(args.steps):
        b = args.warmup + i
        step(b, dev_batches[b])
        stats["m"].append(0)
    t_end.record()
    barrier()
    gv_b200.profile_enable(False)
    launches = gv_b200.kernel_launches() - launches0
    clocks = sampler.stop(h_start, time.monotonic())
    elapsed_ms = t_start.elapsed_time(t_end)
    timed_sweeps = list(stats["pr_sweeps"])  # the e2e leg below appends its own
    m_now = g.num_edges()
    try:
        tc_work = g.last_stat("tc_work")
        tc_probes = g.last_stat("tc_probes")
        tc_core = g.last_stat("tc_core")
    except Exception:
        tc_work = tc_probes = tc_core = None
    prof = {s: gv_b200.profile_query(s) for s in gv_b200.PROFILE_SLOTS}

    # e2e: same steps through the C-ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        pin = []
        for b in range(args.warmup + args.steps, total_steps):
            pin.append(tuple(torch.from_numpy(a.astype(np.uint32).view(np.int32)).pin_memory().numpy().view(np.uint32)
                             for a in batches[b]))
        host_out = {"x": torch.empty(n, dtype=torch.float32).pin_memory().numpy(),
                    "bc": torch.empty(n, dtype=torch.float32).pin_memory().numpy()}
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for i, inputs in enumerate(pin):
            step(args.warmup + args.steps + i, inputs, host_out)
        e1.record()
        barrier()
        e2e_ms = e0.elapsed_time(e1)
        n_bc = sum(1 for i in range(len(pin)) if ((args.warmup + args.steps + i) % args.bc_every) == args.bc_every - 1)
        h2d = args.batch * 8  # (src, dst) uint32 per update
        d2h = n * 4 + 8 + (n * 4 * n_bc) // max(1, len(pin))
        e2e = {"ms": e2e_ms, "h2d": h2d, "d2h": d2h}

    # incremental triangle counts (single GPU): batches alternate between
    # gv_update_tc (exact delta) and update + whole-graph count, at the step's
    # batch size and at 1/16 of it (the first inserts and deletes of a batch)
    incr = None
    if n_incr:
        incr = {"exact": True, "sizes": {}}
        # untimed first call: sizes gv_update_tc's scratch like the warm-up steps do for the step
        g.update_tc(*dev_batches[total_steps + 2 * n_incr], compact=True)
        _, t_ref = g.static_tc(per_vertex=False)
        for fi, frac in enumerate((1, 16)):
            k = args.batch // 2 // frac
            rec = {"updates": 2 * k, "update_tc_ms": [], "update_then_static_tc_ms": []}
            for j in range(n_incr):
                ins_s, ins_d, del_s, del_d = (a[:k] for a in dev_batches[total_steps + fi * n_incr + j])
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                if j % 2 == 0:
                    dt, _ = g.update_tc(ins_s, ins_d, del_s, del_d, compact=True)
                    torch.cuda.synchronize()
                    rec["update_tc_ms"].append((time.perf_counter() - t0) * 1e3)
                    _, t_chk = g.static_tc(per_vertex=False)
                    incr["exact"] = incr["exact"] and (t_chk == t_ref + dt)
                    t_ref = t_chk
                else:
                    g.batch_insert(ins_s, ins_d)
                    g.batch_delete(del_s, del_d)
                    g.compaction()
                    _, t_ref = g.static_tc(per_vertex=False)
                    torch.cuda.synchronize()
                    rec["update_then_static_tc_ms"].append((time.perf_counter() - t0) * 1e3)
            incr["sizes"][str(2 * k)] = {"update_tc_ms": statistics.mean(rec["update_tc_ms"]),
                                         "update_then_static_tc_ms": statistics.mean(rec["update_then_static_tc_ms"])}
        incr["triangles_after"] = int(t_ref)
    elapsed_ms, e2e_ms = max_over_ranks([elapsed_ms, e2e["ms"] if e2e else 0.0], dev, dist)
    g.close()
    if rank != 0:
        return

    updates = args.batch * args.steps * world
    value = updates / (elapsed_ms / 1e3)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    # dominant kernel and its roofline
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    avg_sweeps = sum(timed_sweeps) / max(1, len(timed_sweeps))
    alg = None
    if dom == "pull":
        alg = 4 * m_now + 12 * n  # neighbour ids + read x, read 1/deg, write x' per sweep
        unit_note = "4*m + 12*n bytes per sweep"
    elif dom == "tc_count" and tc_work:
        alg = 4 * tc_work  # merged list entries, 4 B each
        unit_note = "4 * sum over merged oriented edges of (|N+(u)| + |N+(v)|) bytes per launch"
    elif dom == "tc_probe" and tc_probes:
        alg = 2 * tc_probes  # 16-bit core-list entries, each tested against a staged row
        unit_note = "2 bytes per core-list entry tested per launch"
    roof = None
    if alg and dom_n:
        per_launch_s = dom_ms / dom_n / 1e3
        achieved = alg / per_launch_s / 1e9
        traffic = None
        tfile = ROOT / "profiles" / "ncu_traffic.json"
        if tfile.exists():
            tj = json.loads(tfile.read_text())
            if dom in tj and tj[dom].get("bytes_per_unit"):
                units = {"pull": m_now, "tc_count": tc_work, "tc_probe": tc_probes}[dom]
                traffic = tj[dom]["bytes_per_unit"] * units
        if dom == "pull":  # the variant that counts the gathered ranks as well
            roof_extra = {"achieved_8m_12n": (8 * m_now + 12 * n) / per_launch_s / 1e9}
        else:
            roof_extra = {}
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": traffic, "algorithmic_bytes": alg,
                "avg_launch_ms": dom_ms / dom_n, "launches": dom_n, "peak_source": peak_src,
                "note": unit_note + f"; fraction of {peak_src} HBM copy bandwidth", **roof_extra}
    pr_ms = prof["pull"][0]
    pr_gteps = (m_now * sum(timed_sweeps)) / (pr_ms / 1e3) / 1e9 if pr_ms else None
    # betweenness calls in the timed region: TEPS = m * sources / device time
    bc_calls = sum(1 for i in range(args.steps) if ((args.warmup + i) % args.bc_every) == args.bc_every - 1)
    bc_ms = prof["bfs_level"][0] + prof["bc_dep"][0]
    bc_info = None
    if bc_calls and bc_ms:
        bc_info = {"sources": args.bc_sources, "calls": bc_calls, "ms_per_call": bc_ms / bc_calls,
                   "forward_ms_per_call": prof["bfs_level"][0] / bc_calls,
                   "dependency_ms_per_call": prof["bc_dep"][0] / bc_calls,
                   "gteps": m_now * args.bc_sources * bc_calls / (bc_ms / 1e3) / 1e9}
    phases = {k: {"ms_total": v[0], "launches": v[1]} for k, v in prof.items() if v[1]}
    line = {"metric": METRIC, "value": value, "unit": "edge updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded R-MAT graph, uniform-random inserts, deletes sampled from existing edges)",
            "config": workload_config(args, n, m0),
            "pagerank_gteps": pr_gteps, "pagerank_sweeps_avg": avg_sweeps, "m_entries": m_now,
            "betweenness": bc_info,
            "triangles": {"merged_entries": tc_work, "core_probes": tc_probes, "core_vertices": tc_core},
            "kernel_ms": phases, "roofline": roof, "gpu_launches": launches, "clocks": clocks}
    if incr:
        line["incremental_tc"] = {
            "workload": ("same graph as the steps, batches of the step's size and of 1/16 of it; gv_update_tc "
                         "(inserts, deletes, compaction and the exact triangle delta) against insert + delete + "
                         "compaction + whole-graph count"),
            "by_batch_updates": incr["sizes"], "exact": incr["exact"], "triangles_after": incr["triangles_after"]}
    if e2e:
        line["e2e"] = {"value": updates / (e2e_ms / 1e3), "unit": "edge updates/s",
                       "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]}
    if world == 1 and not args.no_batching:
        line["batching"] = run_batching(args, torch.device("cuda", local_rank))
    if world == 1 and not args.no_ingest:
        line["ingest"] = run_ingest(args)
    if world == 1 and not args.no_diff:
        line["differentiation"] = run_differentiation(args)
    if world == 1 and not args.no_serving:
        line["serving"] = run_serving(args, torch.device("cuda", local_rank))
    if world == 1 and not args.no_cpu_baseline:
        import gv_b200 as gvb
        pairs = gvb.gen_rmat(args.scale, args.edge_factor << args.scale, seed)
        threads = os.cpu_count() or 1
        step_s, detail = cpu_sample(args, pairs, batches[:1], n, threads, 1)
        line["cpu_baseline"] = {"value": args.batch / step_s, "unit": "edge updates/s", "cores": threads,
                                "kind": "port",
                                "sample": (f"oracle port (C++/OpenMP): 1 full step (1M updates, PageRank, TC) on the "
                                           f"same graph; BC timed on 4 of {args.bc_sources} sources, scaled and "
                                           f"amortised over {args.bc_every} steps"),
                                "phases_s": detail}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_gv(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
