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
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle comparison of the final graph")
    ap.add_argument("--repeats", type=int, default=3, help="timed repeats of the K steps (median reported)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-batching", action="store_true", help="skip the scale-24 batched-vs-plain section")
    ap.add_argument("--batch-scale", type=int, default=24)
    ap.add_argument("--c3-batches", type=int, default=64)
    ap.add_argument("--no-autotune", action="store_true", help="batching section: use --block/--tpv, skip the autotuner")
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
    ap.add_argument("--serve-ppr-batch", type=int, default=32, help="most PPR queries per served job")
    ap.add_argument("--serve-load", type=float, default=0.7, help="Poisson rate as a fraction of served capacity")
    ap.add_argument("--serve-hbm", type=int, default=96, help="GB of HBM the serving loop may give queries")
    ap.add_argument("--serve-parity-prefix", type=int, default=40,
                    help="requests of the trace replayed with exact epochs and compared with the plain run")
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

    def stop(self, windows=None) -> dict | None:
        """Summary of the samples taken inside the timed windows [(t0, t1), ...]
        (host monotonic time; all samples when none falls inside them)."""
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
        inside = [ln for t, ln in self.lines if any(t0 <= t <= t1 + 0.2 for t0, t1 in (windows or []))]
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
def make_batches(n, off, dst, steps, half, seed, uniform):
    """Per step: uniform new pairs to insert (uniform(n, count, seed) -> (src,
    dst), libgv's or the oracle's copy of the same generator), existing
    undirected edges to delete."""
    deg = np.diff(off).astype(np.int64)
    src_of = np.repeat(np.arange(n, dtype=np.uint32), deg)
    und = np.nonzero(src_of < dst)[0]  # each undirected edge once
    rng = np.random.default_rng(seed)
    picks = rng.choice(len(und), size=min(len(und), steps * half), replace=False)
    out = []
    for b in range(steps):
        ins_s, ins_d = uniform(n, half, seed * 1000 + b)
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
BC_SAMPLE = 4  # BC sources per CPU step (the GPU step runs 64 every 5 steps)


def cpu_step(args, g, batch, src):
    """One step of the workload on the oracle graph `g`: the batch's inserts
    and deletes, PageRank, the triangle total and BC from `src`.  Returns
    (seconds, phase seconds)."""
    ins_s, ins_d, del_s, del_d = batch
    t0 = time.perf_counter()
    g.insert(ins_s, ins_d)
    g.delete(del_s, del_d)
    t1 = time.perf_counter()
    g.pagerank(ALPHA, EPS, MAX_ITER)
    t2 = time.perf_counter()
    g.tc(per_vertex=False)
    t3 = time.perf_counter()
    g.bc(src)
    t4 = time.perf_counter()
    return t4 - t0, {"update_s": t1 - t0, "pagerank_s": t2 - t1, "tc_s": t3 - t2, f"bc_{len(src)}src_s": t4 - t3}


def cpu_sample_note(args, threads, steps):
    return (f"oracle port (C++/OpenMP, {threads} threads), {steps} step(s) of the workload, each: the step's "
            f"{args.batch} updates, PageRank and the triangle total in full, and BC from {BC_SAMPLE} of the "
            f"{args.bc_sources} sources (the GPU step runs {args.bc_sources} sources every {args.bc_every} steps, "
            f"{args.bc_sources / args.bc_every:.1f} per step on average, so this sample does less BC work than "
            f"a GPU step); nothing extrapolated")


def run_reference(args, rank, world):
    """The reference's semantics on the host's cores (the reference has no CPU
    path, so this is the oracle port): the same graph, batches and step
    sequence as the GPU arm; warm-up steps apply their updates only."""
    if rank != 0:
        return
    import oracle
    n = 1 << args.scale
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    pairs = oracle.rmat_pairs(args.scale, args.edge_factor << args.scale, args.seed)
    g = oracle.OracleGraph(n)
    g.insert(*pairs)
    del pairs
    off, dst, _ = g.export()
    m0 = int(off[-1])
    batches = make_batches(n, off, dst, args.warmup + args.steps, args.batch // 2, args.seed, oracle.uniform_pairs)
    del off, dst
    src = bc_sources(n, args.bc_sources, args.seed)[:BC_SAMPLE]
    for b in range(args.warmup):
        g.insert(*batches[b][:2])
        g.delete(*batches[b][2:])
    times, phases = [], []
    for i in range(args.steps):
        t, ph = cpu_step(args, g, batches[args.warmup + i], src)
        times.append(t)
        phases.append(ph)
    total = sum(times)
    value = args.batch * args.steps / total
    line = {"metric": METRIC, "value": value, "unit": "edge updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded R-MAT, uniform inserts, sampled deletes)", "impl": "reference",
            "config": workload_config(args, n, m0),
            "cpu_baseline": {"value": value, "unit": "edge updates/s", "cores": threads, "kind": "port",
                             "sample": cpu_sample_note(args, threads, args.steps),
                             "phases_s_median": {k: statistics.median(p[k] for p in phases) for k in phases[0]}},
            "e2e": {"value": value, "unit": "edge updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- parity
def _mix64(z):
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def adjacency_digest(off, dst, chunk=1 << 24):
    """Order-independent digest of a CSR adjacency: the degree array and two
    commutative 64-bit folds (wrapping sum and xor) of a mixed (u, v) key per
    entry, so two stores with equal digests hold the same neighbour sets up
    to a 2^-64-scale collision."""
    n = len(off) - 1
    deg = np.diff(off.astype(np.int64))
    src = np.repeat(np.arange(n, dtype=np.uint64), deg)
    h_sum, h_xor = np.uint64(0), np.uint64(0)
    with np.errstate(over="ignore"):
        for i in range(0, len(dst), chunk):
            k = (src[i:i + chunk] << np.uint64(32)) | dst[i:i + chunk].astype(np.uint64)
            h_sum = h_sum + _mix64(k).sum(dtype=np.uint64)
            h_xor = h_xor ^ np.bitwise_xor.reduce(_mix64(k ^ np.uint64(0x5851F42D4C957F2D)))
    return deg, int(h_sum), int(h_xor)


def bc_errors(got, want):
    """max relative error over vertices with a nonzero fp64 score, and the
    largest |score| where the fp64 score is zero"""
    got = got.astype(np.float64)
    nz = want != 0
    rel = float(np.max(np.abs(got[nz] - want[nz]) / np.abs(want[nz]))) if nz.any() else 0.0
    zero_abs = float(np.max(np.abs(got[~nz]))) if (~nz).any() else 0.0
    return rel, zero_abs


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


def update_alg_bytes(deg, pairs_src, pairs_dst, del_src, del_dst):
    """Algorithmic bytes of applying one batch of undirected updates: 8 B per
    input pair, one read of every touched vertex's adjacency plus 16 B of its
    metadata, 4 B per directed entry written or tombstoned (2 per pair), and
    a read and write of every vertex with deletes during compaction."""
    touched = np.unique(np.concatenate([pairs_src, pairs_dst]))
    dtouch = np.unique(np.concatenate([del_src, del_dst]))
    p = len(pairs_src)
    return 8 * p + int((4 * deg[touched] + 16).sum()) + 4 * 2 * p + int((8 * deg[dtouch]).sum())


def run_batching(args, dev, hbm_peak):
    """Batching workload: 64 uneven Zipf batches on R-MAT scale 24, plain
    (one synchronous call per batch + compaction, as the reference) against
    the batched window; 32 PPR queries one by one against one batched call."""
    import torch
    import gv_b200
    scale = args.batch_scale
    n = 1 << scale
    seed = args.seed + 100
    # autotune on a scale-20 sample of the same workload shape
    if args.no_autotune:
        best, tune = {"block_size": args.block, "threads_per_vertex": args.tpv}, []
    else:
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
    deg0 = np.diff(off.astype(np.int64))
    del off, dst
    # algorithmic bytes with the initial degrees: per batch (the plain calls)
    # and once over the window (what the batched form must at least move)
    alg_plain = sum(update_alg_bytes(deg0, np.concatenate([a, c]), np.concatenate([b_, e]), c, e)
                    for a, b_, c, e in batches)
    alg_window = update_alg_bytes(deg0, np.concatenate([np.concatenate([a, c]) for a, b_, c, e in batches]),
                                  np.concatenate([np.concatenate([b_, e]) for a, b_, c, e in batches]),
                                  np.concatenate([c for a, b_, c, e in batches]),
                                  np.concatenate([e for a, b_, c, e in batches]))
    del deg0
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
    # capture the window graph of this capacity ahead of the timed window: a
    # window of the same size made of self-loops, which change nothing
    loops = (torch.arange(tot, device=dev, dtype=torch.int64) % n).to(torch.int32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gb.batch_run(([(0, tot, 0)], loops, loops), compact=True, graph=True)
    gb.synchronize()
    capture_s = time.perf_counter() - t0
    del loops
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
    # the batched window must leave exactly the graph the batch-by-batch calls left
    po, pd_, _ = gp.export_csr()
    dig_p = adjacency_digest(po, pd_)
    del po, pd_
    bo, bd, _ = gb.export_csr()
    dig_b = adjacency_digest(bo, bd)
    del bo, bd
    same_graph = bool(np.array_equal(dig_p[0], dig_b[0])) and dig_p[1:] == dig_b[1:]
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
    # 8 queries: one at a time against one batched call over the sweep plan
    x8 = torch.empty((n, 8), dtype=torch.float32, device=dev)
    e[0].record()
    for sq in srcs_q[:8]:
        gp.ppr(int(sq), out=xq)
    e[1].record()
    e[2].record()
    _, sw_8 = gb.ppr_batch(srcs_q[:8], out=x8)
    e[3].record()
    torch.cuda.synchronize()
    pr8 = {"plain_ms": e[0].elapsed_time(e[1]), "batched_ms": e[2].elapsed_time(e[3]), "sweeps": sw_8,
           "max_query_l1_vs_32_batch": float((x8.double() - xb[:, :8].double()).abs().sum(0).max())}
    pr8["speedup"] = pr8["plain_ms"] / pr8["batched_ms"]
    del x8
    gteps_plain = m_p * sw_plain / (pr_plain_ms / 1e3) / 1e9
    gteps_batched = m_b * sw_b * 32 / (pr_batched_ms / 1e3) / 1e9
    # PPR bytes: per single-query sweep 4m + 12n; per batched sweep of k
    # queries 4m + 8kn (the n x k iterate read and written) + 4n
    ppr_alg_plain = sw_plain * (4 * m_p + 12 * n)
    ppr_alg_batched = sw_b * (4 * m_b + 8 * 32 * n + 4 * n)
    gb_stats = {k: gb.last_stat(k) for k in ("window_persistent", "window_exact", "window_captures",
                                             "window_replays")}
    gp.close()
    gb.close()
    del xq
    torch.cuda.empty_cache()
    # the window and the 32 queries as one replayed graph (gv_batch_run_ppr) on
    # a third copy of the initial graph, captured ahead by a self-loop window
    # of the same capacity with the same queries
    gq = gv_b200.GraphVine(n, **cfg)
    s_dev, d_dev = gv_b200.gen_rmat(scale, args.edge_factor << scale, seed, device=dev)
    insert_chunked(gq, s_dev, d_dev)
    del s_dev, d_dev
    loops = (torch.arange(tot, device=dev, dtype=torch.int64) % n).to(torch.int32)
    xw = torch.empty((n, 32), dtype=torch.float32, device=dev)
    gq.batch_run_ppr(([(0, tot, 0)], loops, loops), srcs_q, compact=True, graph=True, out=xw)
    del loops
    torch.cuda.synchronize()
    e[0].record()
    _, sw_w = gq.batch_run_ppr((descs, wsrc, wdst), srcs_q, compact=True, graph=True, out=xw)
    e[1].record()
    torch.cuda.synchronize()
    wq_ms = e[0].elapsed_time(e[1])
    wq_l1 = float((xw.double() - xb.double()).abs().sum(0).max())
    # The two runs sum in different orders (the window's sweeps walk the
    # store, the separate call sweeps the plan) and stop at different sweeps;
    # each stops on an L1 step below epsilon, so each is within
    # epsilon * alpha / (1 - alpha) of the fixed point.
    wq_tol = 2 * EPS * ALPHA / (1 - ALPHA)
    wq_tol_note = "2 eps alpha / (1 - alpha): each result within eps alpha / (1 - alpha) of the fixed point"
    wq_stats = {k: gq.last_stat(k) for k in ("window_captures", "window_replays")}
    gq.close()
    del xw, xb
    torch.cuda.empty_cache()
    window_queries = {
        "what": ("gv_batch_run_ppr: the same window and the same 32 PPR queries as one replayed CUDA graph "
                 "(window, item lists, sweeps and result on the device, no host round trip between them)"),
        "ms": wq_ms, "sweeps": sw_w, "plain_ms": plain_ms + pr_plain_ms,
        "speedup_vs_plain": (plain_ms + pr_plain_ms) / wq_ms,
        "separate_batched_ms": batched_ms + pr_batched_ms,
        "max_query_l1_vs_separate_calls": wq_l1, "tolerance_l1": wq_tol, "tolerance_note": wq_tol_note,
        "ok": wq_l1 <= wq_tol, "graphs": wq_stats}
    return {"workload": (f"R-MAT scale {scale} ef {args.edge_factor}, {len(batches)} batches log-uniform in "
                         f"[1K, 4M] updates, Zipf(1.1) sources, insert fraction U[0.2, 0.8]; 32 PPR queries"),
            "m_initial_entries": m0, "updates": tot, "edges_after_plain": m_p, "edges_after_batched": m_b,
            "plain_updates_per_s": tot / (plain_ms / 1e3), "batched_updates_per_s": tot / (batched_ms / 1e3),
            "updates_speedup": plain_ms / batched_ms,
            "plain": "one synchronous insert, delete and compaction call per batch",
            "batched": ("gv_batch_run: the window reduced to its net effect, one persistent launch applies "
                        "every touched vertex, compaction once; the window's CUDA graph (captured by an earlier "
                        "window of the same capacity, untimed) is replayed"),
            "batched_window_path": gb_stats,
            "capture_window_s": capture_s,
            "pagerank_gteps_plain": gteps_plain, "pagerank_gteps_batched": gteps_batched,
            "pagerank_speedup": pr_plain_ms / pr_batched_ms,
            "pagerank_8_queries": pr8,
            "roofline": {
                "unit": "GB/s", "peak": hbm_peak,
                "updates_plain": {"algorithmic_bytes": alg_plain, "achieved": alg_plain / plain_ms / 1e6,
                                  "frac": alg_plain / plain_ms / 1e6 / hbm_peak},
                "updates_batched": {"algorithmic_bytes": alg_window, "achieved": alg_window / batched_ms / 1e6,
                                    "frac": alg_window / batched_ms / 1e6 / hbm_peak,
                                    "plain_bytes_over_batched_time_frac": alg_plain / batched_ms / 1e6 / hbm_peak},
                "ppr_plain": {"algorithmic_bytes": ppr_alg_plain, "achieved": ppr_alg_plain / pr_plain_ms / 1e6,
                              "frac": ppr_alg_plain / pr_plain_ms / 1e6 / hbm_peak},
                "ppr_batched": {"algorithmic_bytes": ppr_alg_batched,
                                "achieved": ppr_alg_batched / pr_batched_ms / 1e6,
                                "frac": ppr_alg_batched / pr_batched_ms / 1e6 / hbm_peak},
                "note": ("update bytes per batch: 8 per pair + (4 deg + 16) per touched vertex + 8 per pair "
                         "written + 8 deg per vertex with deletes (initial degrees); the window counts each "
                         "touched vertex once")},
            "window_and_queries": window_queries,
            "parity": {"same_graph_as_batch_by_batch": same_graph, "entries": int(dig_p[0].sum()),
                       "tolerance": "bit-exact (degrees + order-independent digests)",
                       "window_queries_max_l1_vs_separate_calls": wq_l1,
                       "window_queries_tolerance_l1": wq_tol, "window_queries_ok": wq_l1 <= wq_tol},
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
    dense = dense_gradient_check(12, seed)
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
                         "tolerance": 1e-4, "oracle_seconds": fd_s,
                         "fd_method": ("perturbed objectives evaluated exactly through the rank-one form of the "
                                       "perturbed fixed point (one fp64 forward-direction solve per edge)")},
            "dense_check": dense}


def dense_gradient_check(scale, seed):
    """The GPU gradient on a directed weighted R-MAT instance small enough for
    dense fp64 solves of the forward and transposed systems (numpy)."""
    import gv_b200
    n = 1 << scale
    rng = np.random.default_rng(seed + scale)
    s, d = gv_b200.gen_rmat(scale, 16 << scale, seed + scale)
    w = (1.0 - 0.9 * rng.random(len(s))).astype(np.float32)
    g = gv_b200.GraphVine(n, directed=True, weighted=True, hbm_budget_bytes=1 << 30)
    g.batch_insert(s, d, w)
    g.synchronize()
    off, dst, wt = g.export_csr(with_weights=True)
    src = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
    Wm = np.zeros((n, n))
    Wm[src, dst] = wt.astype(np.float64)
    rs = Wm.sum(1)
    P = np.divide(Wm, rs[:, None], out=np.zeros_like(Wm), where=rs[:, None] > 0)
    x = np.linalg.solve(np.eye(n) - ALPHA * P.T, np.full(n, (1 - ALPHA) / n))
    c = rng.standard_normal(n)
    lam = np.linalg.solve(np.eye(n) - ALPHA * P, c)
    want = ALPHA * x[src] * (lam[dst] - (P @ lam)[src]) / rs[src]
    xg, _ = g.wpr_forward(ALPHA, 1e-9, 300)
    grad, _, _ = g.wpr_backward(xg, c.astype(np.float32), ALPHA, 1e-9, 300, mode=0)
    g.close()
    return {"scale": scale, "entries": int(len(dst)),
            "forward_l1_vs_dense": float(np.abs(xg.astype(np.float64) - x).sum()),
            "max_err_over_max_grad": float(np.abs(grad.astype(np.float64) - want).max() / np.abs(want).max()),
            "tolerance": 1e-4}


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


def run_serving(args, dev, hbm_peak):
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
    # (the queries of the first `prefix` requests are also kept on the host
    # for the parity sample below)
    prefix = min(len(items), args.serve_parity_prefix)
    kept = {}
    g = build()
    m0 = g.num_edges()
    deg0 = g.degrees().astype(np.int64)
    upd_alg = sum(update_alg_bytes(deg0, np.concatenate([it[1], it[3]]), np.concatenate([it[2], it[4]]),
                                   it[3], it[4]) for it in items if it[0] == "update")
    del deg0
    xq = torch.empty(n, dtype=torch.float32, device=dev)
    bq = torch.empty(n, dtype=torch.float32, device=dev)
    lib = gv_b200._lib.lib()
    t_kind = {"update": 0.0, "ppr": 0.0, "tc": 0.0, "bc": 0.0}
    ppr_edges = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    keep_s = 0.0
    for i, it in enumerate(items):
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
            tcv = g.tc_subset(it[1])
        else:
            src = torch.from_numpy(np.ascontiguousarray(it[1], np.uint32).view(np.int32)).to(dev)
            gv_b200._check(lib.gv_bc(g._h, src.data_ptr(), len(src), bq.data_ptr(), gv_b200.GV_MEM_DEVICE, 0),
                           "gv_bc")
            torch.cuda.synchronize()
        tb = time.perf_counter()
        t_kind[it[0]] += tb - ta
        if i < prefix and it[0] != "update":  # host copies for the parity sample, not counted
            kept[i] = xq.cpu().numpy() if it[0] == "ppr" else (tcv if it[0] == "tc" else bq.cpu().numpy())
            if it[0] == "ppr":
                kept[i] = (kept[i], sw)
            keep_s += time.perf_counter() - tb
    plain_s = time.perf_counter() - t0 - keep_s
    g.close()

    # served, everything arrived at t = 0
    def trace(arrivals, upto=None):
        return [it + (float(a),) for it, a in zip(items[:upto], arrivals)]

    # parity sample: the first `prefix` requests through the loop with exact
    # epochs (each query sees exactly the updates before it, as in the plain
    # run), every query result against the plain run's
    parity = None
    if prefix:
        g = build()
        res_p, outs_p = g.serve(trace(np.zeros(prefix), prefix), slots=args.serve_slots, ppr_batch=args.serve_ppr_batch,
                                pace=False, alpha=ALPHA, epsilon=EPS, max_iter=MAX_ITER,
                                hbm_budget_bytes=args.serve_hbm << 30, outputs=True, fresh=False)
        g.close()
        pr_l1, pr_sw, tc_eq, bc_rel = [], [], [], []
        for i, v in kept.items():
            if items[i][0] == "ppr":
                pr_l1.append(float(np.abs(outs_p[i].astype(np.float64) - v[0]).sum()))
                pr_sw.append((int(res_p["sweeps"][i]), int(v[1])))
            elif items[i][0] == "tc":
                tc_eq.append(bool(np.array_equal(outs_p[i], v)))
            else:
                ref = v.astype(np.float64)
                nz = ref != 0
                bc_rel.append(float(np.max(np.abs(outs_p[i][nz] - ref[nz]) / np.abs(ref[nz]))) if nz.any() else 0.0)
        parity = {"requests": prefix, "fresh": False, "statuses_ok": bool(np.all(res_p["status"] == 0)),
                  "ppr_l1_vs_alone": pr_l1, "ppr_sweeps_served_alone": pr_sw, "tc_equal": tc_eq,
                  "bc_max_rel_vs_alone": bc_rel,
                  "tolerance": "PPR L1 <= 1e-6 (+1e-6 per sweep of difference), TC bit-exact, BC max-rel <= 1e-5",
                  "ok": bool(np.all(res_p["status"] == 0)) and all(tc_eq) and all(r <= 1e-5 for r in bc_rel)
                  and all(l1 <= 1e-6 * (1 + abs(a - b)) for l1, (a, b) in zip(pr_l1, pr_sw))}
        del kept

    g = build()
    t0 = time.perf_counter()
    res, _ = g.serve(trace(np.zeros(len(items))), slots=args.serve_slots, ppr_batch=args.serve_ppr_batch, pace=False,
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
              "update_engine_hbm_frac": upd_alg / max(group_time(res, "update"), 1e-9) / 1e9 / hbm_peak,
              "ppr_gteps": ppr_edges_served / max(group_time(res, "ppr"), 1e-9) / 1e9,
              "groups": int(len(np.unique(res["group"])))}
    plain = {"makespan_s": plain_s, "requests_per_s": len(items) / plain_s, "updates_per_s": upd_pairs / plain_s,
             "update_engine_updates_per_s": upd_pairs / max(t_kind["update"], 1e-9),
             "update_engine_hbm_frac": upd_alg / max(t_kind["update"], 1e-9) / 1e9 / hbm_peak,
             "ppr_gteps": ppr_edges / max(t_kind["ppr"], 1e-9) / 1e9,
             "seconds_by_kind": t_kind}

    # paced: Poisson arrivals at a fraction of the served capacity
    rate = args.serve_load * len(items) / served_s
    arr = np.cumsum(np.random.default_rng(seed + 1).exponential(1.0 / rate, len(items)))
    arr -= arr[0]
    g = build()
    res, _ = g.serve(trace(arr), slots=args.serve_slots, ppr_batch=args.serve_ppr_batch, pace=True, alpha=ALPHA, epsilon=EPS,
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
            "update_algorithmic_bytes": upd_alg,
            "update_bytes_note": ("per update request: 8 per pair + (4 deg + 16) per touched vertex + 8 per pair "
                                  "written + 8 deg per vertex with deletes (initial degrees); the engine fraction "
                                  "divides them by the update requests' time over the measured HBM peak"),
            "plain": plain, "served": served, "parity": parity,
            "served_vs_plain": {"requests": plain_s / served_s,
                                "updates_per_s": served["updates_per_s"] / plain["updates_per_s"],
                                "ppr_gteps": served["ppr_gteps"] / plain["ppr_gteps"] if plain["ppr_gteps"] else None},
            "ppr_batch": args.serve_ppr_batch,
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
    W, K = args.warmup, args.steps
    s_dev, d_dev = gv_b200.gen_rmat(args.scale, args.edge_factor << args.scale, seed, device=dev)

    def build_graph():
        """The initial graph of every repeat: the seeded R-MAT pairs inserted."""
        g = gv_b200.GraphVine(n, block_size=args.block, threads_per_vertex=args.tpv, device=local_rank,
                              max_batch_pairs=args.batch)
        g.batch_insert(s_dev, d_dev)
        g.synchronize()
        return g

    g = build_graph()
    off, dst, _ = g.export_csr()
    m0 = int(off[-1])
    half = args.batch // 2
    n_incr = 0 if (args.no_incremental or world > 1) else 4
    batches = make_batches(n, off, dst, W + K + 2 * n_incr + (1 if n_incr else 0), half, seed,
                           lambda nn, k, sd: gv_b200.gen_uniform(nn, k, seed=sd))
    del off, dst
    srcs = bc_sources(n, args.bc_sources, seed)
    dev_batches = [tuple(torch.from_numpy(a.astype(np.int32)).to(dev) for a in b) for b in batches]
    x_dev = torch.empty(n, dtype=torch.float32, device=dev)
    bc_dev = torch.empty(n, dtype=torch.float32, device=dev)
    src_dev = torch.from_numpy(srcs.astype(np.int32)).to(dev)
    stats = {"pr_sweeps": [], "triangles": []}

    def step(g, b, inputs, host_out=None):
        ins_s, ins_d, del_s, del_d = inputs
        g.batch_insert(ins_s, ins_d)
        g.batch_delete(del_s, del_d)
        g.compaction()
        _, sw = g.static_pagerank(ALPHA, EPS, MAX_ITER, out=x_dev if host_out is None else host_out["x"])
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

    def warm(g):
        # warm-up steps; a BC call as well when no warm-up step ran one, so the
        # BC scratch is sized before the timed region like everything else
        for b in range(W):
            step(g, b, dev_batches[b])
        if W < args.bc_every:
            g.bc(srcs)

    sampler = ClockSampler(local_rank)
    if not args.no_clocks:
        sampler.start()
    windows = []
    # value: R repeats, each on a freshly built graph: W warm-up steps, then
    # exactly K timed steps with the batches resident in HBM
    reps = []
    for r in range(args.repeats):
        if r:
            g.close()
            g = build_graph()
        warm(g)
        barrier()
        for k in stats:
            stats[k].clear()
        gv_b200.profile_reset()
        gv_b200.profile_enable(True)
        launches0 = gv_b200.kernel_launches()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        barrier()
        h0 = time.monotonic()
        t_start.record()
        for i in range(K):
            step(g, W + i, dev_batches[W + i])
        t_end.record()
        barrier()
        windows.append((h0, time.monotonic()))
        gv_b200.profile_enable(False)
        rec = {"ms": t_start.elapsed_time(t_end), "launches": gv_b200.kernel_launches() - launches0,
               "sweeps": list(stats["pr_sweeps"]), "triangles": list(stats["triangles"]),
               "prof": {sl: gv_b200.profile_query(sl) for sl in gv_b200.PROFILE_SLOTS}, "m": g.num_edges()}
        try:
            rec["tc"] = {k: g.last_stat(k) for k in ("tc_work", "tc_probes", "tc_core")}
        except Exception:
            rec["tc"] = {"tc_work": None, "tc_probes": None, "tc_core": None}
        reps.append(rec)

    # e2e: R repeats of the same steps through the C-ABI, batches from pinned
    # host buffers and results copied back to the host inside the timed region
    e2e_ms = []
    if not args.no_e2e:
        pin = [tuple(torch.from_numpy(a.astype(np.uint32).view(np.int32)).pin_memory().numpy().view(np.uint32)
                     for a in batches[b]) for b in range(W, W + K)]
        host_out = {"x": torch.empty(n, dtype=torch.float32).pin_memory().numpy(),
                    "bc": torch.empty(n, dtype=torch.float32).pin_memory().numpy()}
        for r in range(args.repeats):
            g.close()
            g = build_graph()
            warm(g)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            barrier()
            h0 = time.monotonic()
            e0.record()
            for i, inputs in enumerate(pin):
                step(g, W + i, inputs, host_out)
            e1.record()
            barrier()
            windows.append((h0, time.monotonic()))
            e2e_ms.append(e0.elapsed_time(e1))
        n_bc = sum(1 for i in range(K) if ((W + i) % args.bc_every) == args.bc_every - 1)
        h2d = args.batch * 8  # (src, dst) uint32 per update
        d2h = n * 4 + 8 + (n * 4 * n_bc) // max(1, K)
    clocks = sampler.stop(windows)
    del s_dev, d_dev
    torch.cuda.empty_cache()

    # results on the final graph (initial + W + K batches) for the parity
    # check against the oracle, which replays the same batches on the host
    par_gpu = None
    if world == 1 and not args.no_parity:
        pe, pd, _ = g.export_csr()
        xp, swp = g.static_pagerank(ALPHA, EPS, MAX_ITER)
        pvt, tott = g.static_tc(per_vertex=True)
        bsrc = srcs[:BC_SAMPLE]
        par_gpu = {"digest": adjacency_digest(pe, pd), "x": xp, "sweeps": swp, "tc": pvt, "tc_total": tott,
                   "bc_32": g.bc(bsrc),                                     # one 32-source pass
                   "bc_64": g.bc_multi([bsrc[:BC_SAMPLE // 2], bsrc[BC_SAMPLE // 2:]]),  # one 64-source pass
                   "bc_src": bsrc}
        del pe, pd

    # incremental triangle counts (single GPU): batches alternate between
    # gv_update_tc (exact delta) and update + whole-graph count, at the step's
    # batch size and at 1/16 of it (the first inserts and deletes of a batch)
    incr = None
    if n_incr:
        base_b = W + K
        incr = {"exact": True, "sizes": {}}
        # untimed first call: sizes gv_update_tc's scratch like the warm-up steps do for the step
        g.update_tc(*dev_batches[base_b + 2 * n_incr], compact=True)
        _, t_ref = g.static_tc(per_vertex=False)
        for fi, frac in enumerate((1, 16)):
            k = args.batch // 2 // frac
            rec = {"updates": 2 * k, "update_tc_ms": [], "update_then_static_tc_ms": []}
            for j in range(n_incr):
                ins_s, ins_d, del_s, del_d = (a[:k] for a in dev_batches[base_b + fi * n_incr + j])
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
    # the job is as slow as its slowest replica: max over ranks, per repeat
    rep_ms = max_over_ranks([r["ms"] for r in reps] + e2e_ms, dev, dist)
    val_ms, e2e_ms = rep_ms[:len(reps)], rep_ms[len(reps):]
    g.close()
    if rank != 0:
        return

    med = sorted(range(len(reps)), key=lambda i: val_ms[i])[len(reps) // 2]  # the median repeat
    rep = reps[med]
    elapsed_ms = val_ms[med]
    prof, timed_sweeps, m_now = rep["prof"], rep["sweeps"], rep["m"]
    tc_work, tc_probes, tc_core = rep["tc"]["tc_work"], rep["tc"]["tc_probes"], rep["tc"]["tc_core"]
    updates = args.batch * K * world
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
    bc_calls = sum(1 for i in range(K) if ((W + i) % args.bc_every) == args.bc_every - 1)
    bc_ms = prof["bfs_level"][0] + prof["bc_dep"][0]
    bc_info = None
    if bc_calls and bc_ms:
        bc_info = {"sources": args.bc_sources, "calls": bc_calls, "ms_per_call": bc_ms / bc_calls,
                   "forward_ms_per_call": prof["bfs_level"][0] / bc_calls,
                   "dependency_ms_per_call": prof["bc_dep"][0] / bc_calls,
                   "gteps": m_now * args.bc_sources * bc_calls / (bc_ms / 1e3) / 1e9}
        # algorithmic bytes per source: two passes over the adjacency (4 m
        # each) and sigma, dist and delta read and written (2 n (8 + 4 + 4))
        bc_alg = args.bc_sources * (8 * m_now + 32 * n)
        bc_info["algorithmic_bytes_per_call"] = bc_alg
        bc_info["hbm_frac"] = bc_alg / (bc_ms / bc_calls) / 1e6 / hbm_peak
        bc_info["bytes_note"] = (f"per source 2*(4m) + n*(8 sigma + 4 dist + 4 delta)*2; fraction of "
                                 f"{peak_src} HBM copy bandwidth")
    phases = {k: {"ms_total": v[0], "launches": v[1]} for k, v in prof.items() if v[1]}
    line = {"metric": METRIC, "value": value, "unit": "edge updates/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": elapsed_ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded R-MAT graph, uniform-random inserts, deletes sampled from existing edges)",
            "config": workload_config(args, n, m0),
            "repeats": {"count": len(reps), "kind": "median", "note": (
                "each repeat rebuilds the initial graph, runs the warm-up steps, then times exactly K steps; "
                "value and e2e are the median repeats"),
                "value_ms_per_step": [t / K for t in val_ms], "e2e_ms_per_step": [t / K for t in e2e_ms]},
            "pagerank_gteps": pr_gteps, "pagerank_sweeps_avg": avg_sweeps, "m_entries": m_now,
            "betweenness": bc_info,
            "triangles": {"merged_entries": tc_work, "core_probes": tc_probes, "core_vertices": tc_core},
            "kernel_ms": phases, "roofline": roof, "gpu_launches": rep["launches"], "clocks": clocks}
    if incr:
        line["incremental_tc"] = {
            "workload": ("same graph as the steps, batches of the step's size and of 1/16 of it; gv_update_tc "
                         "(inserts, deletes, compaction and the exact triangle delta) against insert + delete + "
                         "compaction + whole-graph count"),
            "by_batch_updates": incr["sizes"], "exact": incr["exact"], "triangles_after": incr["triangles_after"]}
    if e2e_ms:
        e_med = sorted(e2e_ms)[len(e2e_ms) // 2]
        line["e2e"] = {"value": updates / (e_med / 1e3), "unit": "edge updates/s",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    if world == 1 and not args.no_batching:
        line["batching"] = run_batching(args, torch.device("cuda", local_rank), hbm_peak)
    if world == 1 and not args.no_ingest:
        line["ingest"] = run_ingest(args)
    if world == 1 and not args.no_diff:
        line["differentiation"] = run_differentiation(args)
    if world == 1 and not args.no_serving:
        line["serving"] = run_serving(args, torch.device("cuda", local_rank), hbm_peak)
    if world == 1 and (par_gpu is not None or not args.no_cpu_baseline):
        parity, cpu = cpu_legs(args, n, seed, batches, srcs, par_gpu)
        if parity is not None:
            line["parity"] = {"plain_step_graph": parity}
        if cpu is not None:
            line["cpu_baseline"] = cpu
    # one place for every parity result of the run
    par = line.setdefault("parity", {})
    if "batching" in line:
        par["batching_window"] = line["batching"]["parity"]
    if "differentiation" in line:
        dfd = line["differentiation"]
        par["gradient"] = {"fd_max_err_over_max_fd": dfd["fd_check"]["max_err_over_max_fd"],
                           "dense_scale12_max_err_over_max_grad": dfd["dense_check"]["max_err_over_max_grad"],
                           "tolerance": 1e-4}
    if "serving" in line and line["serving"].get("parity"):
        par["serving_sample"] = line["serving"]["parity"]
    print(json.dumps(line), flush=True)


def cpu_legs(args, n, seed, batches, srcs, par_gpu):
    """The oracle on the host: replays the initial graph and the W + K batches
    the GPU applied, compares the GPU's final results with it (adjacency,
    PageRank, triangles, BC), then times one more step as the CPU baseline."""
    import oracle
    import gv_b200
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    t0 = time.perf_counter()
    o = oracle.OracleGraph(n)
    o.insert(*gv_b200.gen_rmat(args.scale, args.edge_factor << args.scale, seed))
    W, K = args.warmup, args.steps
    for b in range(W + K):
        o.insert(*batches[b][:2])
        o.delete(*batches[b][2:])
    parity = None
    if par_gpu is not None:
        ooff, odst, _ = o.export()
        deg_o, hs_o, hx_o = adjacency_digest(ooff, odst)
        del ooff, odst
        deg_g, hs_g, hx_g = par_gpu["digest"]
        xo, _ = o.pagerank(ALPHA, EPS, MAX_ITER, fixed_sweeps=par_gpu["sweeps"])
        pvo, toto = o.tc(per_vertex=True)
        bsrc = par_gpu["bc_src"]
        bo32 = o.bc(bsrc)
        bo64 = [o.bc(bsrc[:BC_SAMPLE // 2]), o.bc(bsrc[BC_SAMPLE // 2:])]
        r32, z32 = bc_errors(par_gpu["bc_32"], bo32)
        r64 = [bc_errors(par_gpu["bc_64"][i], bo64[i]) for i in range(2)]
        pr_l1 = float(np.abs(par_gpu["x"].astype(np.float64) - xo).sum())
        parity = {
            "workload": (f"final graph of the timed steps (initial R-MAT scale {args.scale} + {W + K} batches of "
                         f"{args.batch} updates) against the oracle replaying the same batches on the host"),
            "adjacency": {"degrees_equal": bool(np.array_equal(deg_g, deg_o)),
                          "digest_equal": (hs_g, hx_g) == (hs_o, hx_o), "entries": int(deg_o.sum()),
                          "tolerance": "bit-exact (degrees + order-independent 64-bit digests of the (u, v) set)"},
            "pagerank": {"l1_vs_fp64": pr_l1, "sweeps": int(par_gpu["sweeps"]), "tolerance_l1": 1e-6,
                         "ok": pr_l1 <= 1e-6},
            "triangles": {"total_gpu": int(par_gpu["tc_total"]), "total_oracle": int(toto),
                          "per_vertex_equal": bool(np.array_equal(par_gpu["tc"], pvo)),
                          "tolerance": "bit-exact (uint64 per vertex, min-id owner)"},
            "betweenness": {"sources": [int(v) for v in bsrc],
                            "pass_32": {"max_rel_vs_fp64": r32, "max_abs_where_fp64_zero": z32},
                            "pass_64_two_requests": {"max_rel_vs_fp64": max(r[0] for r in r64),
                                                     "max_abs_where_fp64_zero": max(r[1] for r in r64)},
                            "tolerance_max_rel": 1e-5},
            "oracle_seconds": time.perf_counter() - t0}
        parity["triangles"]["ok"] = parity["triangles"]["per_vertex_equal"] and (
            parity["triangles"]["total_gpu"] == parity["triangles"]["total_oracle"])
        parity["betweenness"]["ok"] = max(r32, max(r[0] for r in r64)) <= 1e-5 and max(z32, max(r[1] for r in r64)) == 0
        parity["adjacency"]["ok"] = parity["adjacency"]["degrees_equal"] and parity["adjacency"]["digest_equal"]
    cpu = None
    if not args.no_cpu_baseline:
        t, ph = cpu_step(args, o, batches[W + K], srcs[:BC_SAMPLE])
        cpu = {"value": args.batch / t, "unit": "edge updates/s", "cores": threads, "kind": "port",
               "sample": cpu_sample_note(args, threads, 1), "phases_s": ph}
    return parity, cpu


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
