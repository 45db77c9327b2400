"""gv_b200 — B200-native GraphVine dynamic-graph store and analytics.

Python mirror of the reference's host API (class GraphVine in
include/dynamicStructure/graphvine.cuh:29-58 and the algorithm entry points
static_pagerank / dynamic_pagerank / static_tc / dynamic_tc / bc), calling
libgv.so through its C ABI.  Arrays are numpy (host memory) or torch CUDA
tensors (device memory); vertex ids are 0-based uint32.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import GV_MEM_DEVICE, GV_MEM_HOST, GV_OK, STATUS_NAMES, gv_config

__all__ = ["GraphVine", "GvError", "gen_rmat", "gen_uniform", "kernel_launches", "mtx_parse", "version"]


class GvError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = _lib.lib().gv_last_error_string().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")


def _check(st: int, where: str) -> None:
    if st != GV_OK:
        raise GvError(st, where)


def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


def _ptr(a, dtype) -> tuple[int, int, object]:
    """(pointer, mem flag, keep-alive) for a numpy array or a torch CUDA tensor."""
    if a is None:
        return 0, GV_MEM_HOST, None
    if _is_torch_cuda(a):
        import torch
        want = {np.uint32: (torch.int32, torch.uint32), np.float32: (torch.float32,),
                np.uint64: (torch.int64, torch.uint64), np.int32: (torch.int32,), np.uint8: (torch.uint8,)}[dtype]
        if a.dtype not in want:
            raise TypeError(f"device tensor must have dtype {want[0]}, got {a.dtype}")
        if not a.is_contiguous():
            raise ValueError("device tensor must be contiguous")
        return a.data_ptr(), GV_MEM_DEVICE, a
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data, GV_MEM_HOST, arr


def _stream(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


def kernel_launches() -> int:
    return int(_lib.lib().gv_kernel_launches())


def version() -> str:
    return _lib.lib().gv_version().decode()


PROFILE_SLOTS = ("radix", "segment", "member", "apply", "compact", "pull", "tc_snapshot", "tc_count",
                 "bfs_level", "bc_dep", "wpr_build", "wpr_sweep", "wpr_grad", "tc_core", "tc_probe",
                 "tc_sort")


def profile_enable(on: bool = True) -> None:
    _check(_lib.lib().gv_profile_enable(int(on)), "gv_profile_enable")


def profile_reset() -> None:
    _check(_lib.lib().gv_profile_reset(), "gv_profile_reset")


def profile_query(slot: str) -> tuple[float, int]:
    """(total device ms, launches) recorded for a kernel slot since the last reset."""
    ms, n = C.c_double(), C.c_uint64()
    _check(_lib.lib().gv_profile_query(slot.encode(), C.byref(ms), C.byref(n)), "gv_profile_query")
    return ms.value, n.value


def gen_rmat(scale: int, num_pairs: int, seed: int, first: int = 0, device=None, stream=None):
    """R-MAT pairs (src, dst) as numpy arrays, or torch CUDA tensors if device is given."""
    L = _lib.lib()
    if device is not None:
        import torch
        src = torch.empty(num_pairs, dtype=torch.int32, device=device)
        dst = torch.empty(num_pairs, dtype=torch.int32, device=device)
        _check(L.gv_gen_rmat(scale, first, num_pairs, seed, src.data_ptr(), dst.data_ptr(), GV_MEM_DEVICE,
                             _stream(stream)), "gv_gen_rmat")
        return src, dst
    src = np.empty(num_pairs, np.uint32)
    dst = np.empty(num_pairs, np.uint32)
    _check(L.gv_gen_rmat(scale, first, num_pairs, seed, src.ctypes.data, dst.ctypes.data, GV_MEM_HOST, 0), "gv_gen_rmat")
    return src, dst


def gen_uniform(n: int, count: int, seed: int, device=None, stream=None):
    L = _lib.lib()
    if device is not None:
        import torch
        src = torch.empty(count, dtype=torch.int32, device=device)
        dst = torch.empty(count, dtype=torch.int32, device=device)
        _check(L.gv_gen_uniform(n, count, seed, src.data_ptr(), dst.data_ptr(), GV_MEM_DEVICE, _stream(stream)),
               "gv_gen_uniform")
        return src, dst
    src = np.empty(count, np.uint32)
    dst = np.empty(count, np.uint32)
    _check(L.gv_gen_uniform(n, count, seed, src.ctypes.data, dst.ctypes.data, GV_MEM_HOST, 0), "gv_gen_uniform")
    return src, dst


def autotune(num_vertices: int, src0, dst0, batches, *, device: int = 0, hbm_budget_bytes: int = 0,
             max_batch_pairs: int = 1 << 20):
    """Times edge-block size {32, 64, 128} x threads-per-vertex {4, 8, 16, 32}
    on a sample workload (build from src0/dst0, one window of `batches` as in
    GraphVine.batch_run, one PageRank).  Returns (best dict, [results])."""
    L = _lib.lib()
    cfg = gv_config()
    _check(L.gv_config_init(C.byref(cfg), num_vertices), "gv_config_init")
    cfg.device = device
    cfg.hbm_budget_bytes = hbm_budget_bytes
    cfg.max_batch_pairs = max_batch_pairs
    descs, srcs, dsts, off = [], [], [], 0
    for ins_s, ins_d, del_s, del_d in batches:
        descs.append((off, len(ins_s), len(del_s)))
        srcs += [np.asarray(ins_s, np.uint32), np.asarray(del_s, np.uint32)]
        dsts += [np.asarray(ins_d, np.uint32), np.asarray(del_d, np.uint32)]
        off += len(ins_s) + len(del_s)
    bs, bd = np.concatenate(srcs), np.concatenate(dsts)
    s0, d0 = np.ascontiguousarray(src0, np.uint32), np.ascontiguousarray(dst0, np.uint32)
    arr = (_lib.gv_batch_desc * len(descs))(*[_lib.gv_batch_desc(o, i, d) for o, i, d in descs])
    res = (_lib.gv_tune_result * 12)()
    nres = C.c_uint32(12)
    best = gv_config()
    _check(L.gv_autotune(C.byref(cfg), s0.ctypes.data, d0.ctypes.data, len(s0), arr, len(descs), bs.ctypes.data,
                         bd.ctypes.data, GV_MEM_HOST, res, C.byref(nres), C.byref(best)), "gv_autotune")
    results = [{"block_size": r.block_size, "threads_per_vertex": r.threads_per_vertex, "update_ms": r.update_ms,
                "pagerank_ms": r.pagerank_ms} for r in res[:nres.value]]
    return {"block_size": best.block_size, "threads_per_vertex": best.threads_per_vertex}, results


def mtx_parse(text, with_values: bool = False):
    """Parses Matrix-Market coordinate text (bytes, or a torch CUDA uint8
    tensor) on the device: (info dict, src, dst, values or None), 0-based."""
    L = _lib.lib()
    info = _lib.gv_mtx_info()
    cnt = C.c_uint64()
    if _is_torch_cuda(text):
        import torch
        ptr, mem, n = text.data_ptr(), GV_MEM_DEVICE, text.numel()
    else:
        buf = np.frombuffer(bytes(text), dtype=np.uint8)
        ptr, mem, n = buf.ctypes.data, GV_MEM_HOST, len(buf)
    _check(L.gv_mtx_parse(ptr, n, mem, C.byref(info), None, None, None, 0, C.byref(cnt), None), "gv_mtx_parse")
    cap = int(info.entries) + 16
    if mem == GV_MEM_DEVICE:
        import torch
        src = torch.empty(cap, dtype=torch.int32, device=text.device)
        dst = torch.empty(cap, dtype=torch.int32, device=text.device)
        val = torch.empty(cap, dtype=torch.float32, device=text.device) if with_values else None
        ps, pd, pv = src.data_ptr(), dst.data_ptr(), (val.data_ptr() if val is not None else None)
    else:
        src, dst = np.empty(cap, np.uint32), np.empty(cap, np.uint32)
        val = np.empty(cap, np.float32) if with_values else None
        ps, pd, pv = src.ctypes.data, dst.ctypes.data, (val.ctypes.data if val is not None else None)
    _check(L.gv_mtx_parse(ptr, n, mem, C.byref(info), ps, pd, pv, cap, C.byref(cnt), None), "gv_mtx_parse")
    k = cnt.value
    meta = {"rows": info.rows, "cols": info.cols, "entries": info.entries, "pattern": bool(info.pattern),
            "symmetric": bool(info.symmetric)}
    return meta, src[:k], dst[:k], (val[:k] if val is not None else None)


class GraphVine:
    """A dynamic graph resident on one GPU (edge-block CBT store)."""

    def __init__(self, num_vertices: int, *, block_size: int = 128, threads_per_vertex: int = 8,
                 directed: bool = False, weighted: bool = False, device: int = 0, pool_blocks: int = 0,
                 hbm_budget_bytes: int = 0, max_batch_pairs: int = 1 << 20):
        L = _lib.lib()
        cfg = gv_config()
        _check(L.gv_config_init(C.byref(cfg), num_vertices), "gv_config_init")
        cfg.block_size = block_size
        cfg.threads_per_vertex = threads_per_vertex
        cfg.directed = int(directed)
        cfg.weighted = int(weighted)
        cfg.device = device
        cfg.pool_blocks = pool_blocks
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.max_batch_pairs = max_batch_pairs
        h = C.c_void_p()
        _check(L.gv_create(C.byref(cfg), C.byref(h)), "gv_create")
        self._h = h
        self.n = num_vertices
        self.weighted = weighted
        self.directed = directed
        self.device = device

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().gv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    @classmethod
    def _wrap(cls, h: C.c_void_p) -> "GraphVine":
        cfg = gv_config()
        _check(_lib.lib().gv_get_config(h, C.byref(cfg)), "gv_get_config")
        g = cls.__new__(cls)
        g._h, g.n, g.weighted, g.directed, g.device = h, cfg.num_vertices, bool(cfg.weighted), bool(cfg.directed), cfg.device
        return g

    @classmethod
    def from_mtx(cls, path: str, *, weighted: bool = False, directed: bool = False, hbm_budget_bytes: int = 0,
                 block_size: int = 128) -> "GraphVine":
        """Builds a graph from a Matrix-Market file parsed on the device."""
        L = _lib.lib()
        cfg = gv_config()
        _check(L.gv_config_init(C.byref(cfg), 1), "gv_config_init")
        cfg.weighted, cfg.directed, cfg.hbm_budget_bytes, cfg.block_size = int(weighted), int(directed), \
            hbm_budget_bytes, block_size
        h = C.c_void_p()
        _check(L.gv_graph_from_mtx(str(path).encode(), C.byref(cfg), C.byref(h)), "gv_graph_from_mtx")
        return cls._wrap(h)

    @classmethod
    def snapshot_load(cls, path: str, *, hbm_budget_bytes: int = 0) -> "GraphVine":
        """A new graph from a snapshot written by snapshot_save."""
        L = _lib.lib()
        h = C.c_void_p()
        if hbm_budget_bytes:
            cfg = gv_config()
            _check(L.gv_config_init(C.byref(cfg), 1), "gv_config_init")
            cfg.hbm_budget_bytes = hbm_budget_bytes
            _check(L.gv_snapshot_load(str(path).encode(), C.byref(cfg), C.byref(h)), "gv_snapshot_load")
        else:
            _check(L.gv_snapshot_load(str(path).encode(), None, C.byref(h)), "gv_snapshot_load")
        return cls._wrap(h)

    def snapshot_save(self, path: str) -> None:
        _check(_lib.lib().gv_snapshot_save(self._h, str(path).encode()), "gv_snapshot_save")

    def view(self) -> "GraphVine":
        """A read-only view: shares this graph's store and owns its analytics
        scratch, so queries can run on other threads and streams while nothing
        updates the graph.  Close views before the graph."""
        h = C.c_void_p()
        _check(_lib.lib().gv_view_create(self._h, C.byref(h)), "gv_view_create")
        v = GraphVine.__new__(GraphVine)
        v._h, v.n, v.weighted, v.directed, v.device = h, self.n, self.weighted, self.directed, self.device
        v._parent = self
        return v

    # -- updates (GraphVine::bulkBuild / batchInsert / batchDelete / compaction)
    def bulk_build(self, offsets, dst, weights=None, stream=None) -> None:
        po, mem, k1 = _ptr(offsets, np.uint64)
        pd, _, k2 = _ptr(dst, np.uint32)
        pw, _, k3 = _ptr(weights, np.float32)
        _check(_lib.lib().gv_bulk_build_csr(self._h, po, pd, pw or None, mem, _stream(stream)), "gv_bulk_build_csr")

    def batch_insert(self, src, dst, weights=None, stream=None) -> None:
        ps, mem, k1 = _ptr(src, np.uint32)
        pd, _, k2 = _ptr(dst, np.uint32)
        pw, _, k3 = _ptr(weights, np.float32)
        k = len(src)
        _check(_lib.lib().gv_insert_edges(self._h, ps, pd, pw or None, k, mem, _stream(stream)), "gv_insert_edges")
        if mem == GV_MEM_HOST:
            self._keep = (k1, k2, k3)

    def batch_delete(self, src, dst, stream=None) -> None:
        ps, mem, k1 = _ptr(src, np.uint32)
        pd, _, k2 = _ptr(dst, np.uint32)
        _check(_lib.lib().gv_delete_edges(self._h, ps, pd, len(src), mem, _stream(stream)), "gv_delete_edges")
        if mem == GV_MEM_HOST:
            self._keep = (k1, k2)

    def compaction(self, stream=None) -> None:
        _check(_lib.lib().gv_compact(self._h, _stream(stream)), "gv_compact")

    def add_vertices(self, k: int, stream=None) -> int:
        """Adds k isolated vertices; returns the first new id."""
        first = C.c_uint32()
        _check(_lib.lib().gv_add_vertices(self._h, k, C.byref(first), _stream(stream)), "gv_add_vertices")
        self.n += k
        return first.value

    def delete_vertices(self, ids, compact: bool = True, stream=None) -> None:
        """Removes every edge incident to the given vertices (ids stay valid)."""
        pi, mem, keep = _ptr(ids, np.uint32)
        k = len(ids)
        _check(_lib.lib().gv_delete_vertices(self._h, pi, k, 1 if compact else 0, mem, _stream(stream)),
               "gv_delete_vertices")

    def synchronize(self, stream=None) -> None:
        _check(_lib.lib().gv_synchronize(self._h, _stream(stream)), "gv_synchronize")

    # -- batched updates and queries ----------------------------------------
    def batch_run(self, batches, compact: bool = True, graph: bool = False, stream=None) -> None:
        """Apply a window of batches [(ins_src, ins_dst, del_src, del_dst), ...]
        or (descs, src, dst) already laid out; equal to applying them in order."""
        if isinstance(batches, tuple) and len(batches) == 3 and not isinstance(batches[0], tuple):
            descs, src, dst = batches
        else:
            descs, srcs, dsts, off = [], [], [], 0
            for ins_s, ins_d, del_s, del_d in batches:
                descs.append((off, len(ins_s), len(del_s)))
                srcs += [np.asarray(ins_s, np.uint32), np.asarray(del_s, np.uint32)]
                dsts += [np.asarray(ins_d, np.uint32), np.asarray(del_d, np.uint32)]
                off += len(ins_s) + len(del_s)
            src, dst = np.concatenate(srcs), np.concatenate(dsts)
        arr = (_lib.gv_batch_desc * len(descs))(*[_lib.gv_batch_desc(o, i, d) for o, i, d in descs])
        ps, mem, k1 = _ptr(src, np.uint32)
        pd, _, k2 = _ptr(dst, np.uint32)
        flags = (_lib.GV_BATCH_COMPACT if compact else 0) | (_lib.GV_BATCH_GRAPH if graph else 0)
        _check(_lib.lib().gv_batch_run(self._h, arr, len(descs), ps, pd, mem, flags, _stream(stream)), "gv_batch_run")
        self._keep = (k1, k2, arr)

    def batch_run_ppr(self, batches, sources, compact: bool = True, graph: bool = False, alpha: float = 0.85,
                      epsilon: float = 1e-6, max_iter: int = 100, out=None, stream=None):
        """A window of batches (as batch_run takes them), then k <= 32 PPR
        queries on the resulting graph in the same unit of device work
        (gv_batch_run_ppr); returns (x[n, k], sweeps).  out: a device tensor
        when the batches are device tensors, else a host array."""
        if isinstance(batches, tuple) and len(batches) == 3 and not isinstance(batches[0], tuple):
            descs, src, dst = batches
        else:
            descs, srcs, dsts, off = [], [], [], 0
            for ins_s, ins_d, del_s, del_d in batches:
                descs.append((off, len(ins_s), len(del_s)))
                srcs += [np.asarray(ins_s, np.uint32), np.asarray(del_s, np.uint32)]
                dsts += [np.asarray(ins_d, np.uint32), np.asarray(del_d, np.uint32)]
                off += len(ins_s) + len(del_s)
            src = np.concatenate(srcs) if srcs else np.zeros(1, np.uint32)
            dst = np.concatenate(dsts) if dsts else np.zeros(1, np.uint32)
        sv = np.ascontiguousarray(sources, dtype=np.uint32)
        k = len(sv)
        arr = (_lib.gv_batch_desc * max(len(descs), 1))(*[_lib.gv_batch_desc(o, i, d) for o, i, d in descs])
        ps, mem, k1 = _ptr(src, np.uint32)
        pd, _, k2 = _ptr(dst, np.uint32)
        x = np.empty((self.n, k), np.float32) if out is None else out
        px, xmem, _ = _ptr(x, np.float32)
        if xmem != mem:
            raise ValueError("the result must live where the batches do (host or device)")
        sw = C.c_int32()
        flags = (_lib.GV_BATCH_COMPACT if compact else 0) | (_lib.GV_BATCH_GRAPH if graph else 0)
        _check(_lib.lib().gv_batch_run_ppr(self._h, arr, len(descs), ps, pd, mem, flags, sv.ctypes.data, k, alpha,
                                           epsilon, max_iter, px, C.byref(sw), _stream(stream)), "gv_batch_run_ppr")
        self._keep = (k1, k2, arr)
        return x, sw.value

    def ppr_batch(self, sources, alpha: float = 0.85, epsilon: float = 1e-6, max_iter: int = 100, out=None,
                  stream=None):
        """k <= 32 personalised PageRank queries at once; returns (x[n, k], sweeps)."""
        s = np.ascontiguousarray(sources, dtype=np.uint32)
        k = len(s)
        x = np.empty((self.n, k), np.float32) if out is None else out
        px, mem, _ = _ptr(x, np.float32)
        sw = C.c_int32()
        if mem == GV_MEM_DEVICE:
            import torch
            sd = torch.from_numpy(s.view(np.int32)).to(x.device)
            ps = sd.data_ptr()
        else:
            ps = s.ctypes.data
        _check(_lib.lib().gv_ppr_batch(self._h, ps, k, alpha, epsilon, max_iter, px, C.byref(sw), mem,
                                       _stream(stream)), "gv_ppr_batch")
        return x, sw.value

    # -- facts -------------------------------------------------------------
    def num_edges(self) -> int:
        m = C.c_uint64()
        _check(_lib.lib().gv_num_edges(self._h, C.byref(m)), "gv_num_edges")
        return m.value

    def pool_stats(self) -> tuple[int, int]:
        cap, free = C.c_uint64(), C.c_uint64()
        _check(_lib.lib().gv_pool_stats(self._h, C.byref(cap), C.byref(free)), "gv_pool_stats")
        return cap.value, free.value

    def degrees(self) -> np.ndarray:
        out = np.empty(self.n, np.uint32)
        _check(_lib.lib().gv_degrees(self._h, out.ctypes.data, GV_MEM_HOST, 0), "gv_degrees")
        return out

    def export_csr(self, with_weights: bool = False):
        """(offsets[n+1] uint64, dst[m] uint32, weights[m] float32 or None), storage order."""
        m = self.num_edges()
        off = np.empty(self.n + 1, np.uint64)
        dst = np.empty(max(m, 1), np.uint32)
        w = np.empty(max(m, 1), np.float32) if with_weights else None
        _check(_lib.lib().gv_export_csr(self._h, off.ctypes.data, dst.ctypes.data,
                                        w.ctypes.data if w is not None else None, m, GV_MEM_HOST, 0), "gv_export_csr")
        return off, dst[:m], (w[:m] if w is not None else None)

    def affected(self) -> np.ndarray:
        out = np.empty(self.n, np.uint8)
        _check(_lib.lib().gv_affected(self._h, out.ctypes.data, GV_MEM_HOST, 0), "gv_affected")
        return out

    def clear_affected(self, stream=None) -> None:
        _check(_lib.lib().gv_clear_affected(self._h, _stream(stream)), "gv_clear_affected")

    def last_stat(self, key: str) -> float:
        v = C.c_double()
        _check(_lib.lib().gv_last_stat(self._h, key.encode(), C.byref(v)), "gv_last_stat")
        return v.value

    def check(self) -> tuple[int, int, int]:
        v, code, vert = C.c_uint64(), C.c_uint32(), C.c_uint32()
        _check(_lib.lib().gv_check(self._h, C.byref(v), C.byref(code), C.byref(vert)), "gv_check")
        return v.value, code.value, vert.value

    # -- analytics (static_pagerank / dynamic_pagerank / static_tc / bc) ------
    def static_pagerank(self, alpha: float = 0.85, epsilon: float = 1e-6, max_iter: int = 100, out=None, stream=None):
        x = np.empty(self.n, np.float32) if out is None else out
        px, mem, _ = _ptr(x, np.float32)
        sw = C.c_int32()
        _check(_lib.lib().gv_pagerank(self._h, alpha, epsilon, max_iter, px, C.byref(sw), mem, _stream(stream)),
               "gv_pagerank")
        return x, sw.value

    def dynamic_pagerank(self, x, alpha: float = 0.85, epsilon: float = 1e-6, max_iter: int = 100, stream=None):
        """Warm start from x (updated in place for device tensors; returns the result)."""
        if _is_torch_cuda(x):
            px, mem, _ = _ptr(x, np.float32)
            xr = x
        else:
            xr = np.array(x, dtype=np.float32, copy=True)
            px, mem = xr.ctypes.data, GV_MEM_HOST
        sw = C.c_int32()
        _check(_lib.lib().gv_pagerank_dynamic(self._h, alpha, epsilon, max_iter, px, C.byref(sw), mem,
                                              _stream(stream)), "gv_pagerank_dynamic")
        return xr, sw.value

    def ppr(self, source: int, alpha: float = 0.85, epsilon: float = 1e-6, max_iter: int = 100, out=None,
            stream=None):
        x = np.empty(self.n, np.float32) if out is None else out
        px, mem, _ = _ptr(x, np.float32)
        sw = C.c_int32()
        _check(_lib.lib().gv_ppr(self._h, source, alpha, epsilon, max_iter, px, C.byref(sw), mem, _stream(stream)),
               "gv_ppr")
        return x, sw.value

    def static_tc(self, per_vertex: bool = True, stream=None):
        pv = np.empty(self.n, np.uint64) if per_vertex else None
        tot = C.c_uint64()
        _check(_lib.lib().gv_tc(self._h, pv.ctypes.data if pv is not None else None, C.byref(tot), GV_MEM_HOST,
                                _stream(stream)), "gv_tc")
        return pv, tot.value

    def update_tc(self, ins_src, ins_dst, del_src, del_dst, ins_weights=None, compact: bool = True,
                  per_vertex: bool = False, stream=None):
        """Applies inserts, then deletes (then compaction) and returns the exact
        change of the triangle count, and per vertex of its owned triangles
        when per_vertex=True: (delta_total, delta_owner or None)."""
        pis, mem, k1 = _ptr(ins_src, np.uint32)
        pid, _, k2 = _ptr(ins_dst, np.uint32)
        pds, mem2, k3 = _ptr(del_src, np.uint32)
        pdd, _, k4 = _ptr(del_dst, np.uint32)
        pw, _, k5 = _ptr(ins_weights, np.float32)
        if ins_src is None:
            mem = mem2
        elif del_src is not None and mem != mem2:
            raise ValueError("inserts and deletes must live in the same kind of memory")
        ni = len(ins_src) if ins_src is not None else 0
        nd = len(del_src) if del_src is not None else 0
        tot = C.c_int64()
        owner = None
        po = None
        if per_vertex:
            if mem == GV_MEM_DEVICE:
                import torch
                owner = torch.empty(self.n, dtype=torch.int64, device=ins_src.device)
                po = owner.data_ptr()
            else:
                owner = np.empty(self.n, np.int64)
                po = owner.ctypes.data
        _check(_lib.lib().gv_update_tc(self._h, pis, pid, pw, ni, pds, pdd, nd, 1 if compact else 0, C.byref(tot),
                                       po, mem, _stream(stream)), "gv_update_tc")
        return tot.value, owner

    def tc_subset(self, subset, stream=None) -> np.ndarray:
        s = np.ascontiguousarray(subset, dtype=np.uint32)
        out = np.empty(len(s), np.uint64)
        _check(_lib.lib().gv_tc_subset(self._h, s.ctypes.data, len(s), out.ctypes.data, GV_MEM_HOST,
                                       _stream(stream)), "gv_tc_subset")
        return out

    def bc(self, sources=None, stream=None) -> np.ndarray:
        out = np.empty(self.n, np.float32)
        if sources is None:
            ps, ns = None, 0
        else:
            s = np.ascontiguousarray(sources, dtype=np.uint32)
            ps, ns = s.ctypes.data, len(s)
        _check(_lib.lib().gv_bc(self._h, ps, ns, out.ctypes.data, GV_MEM_HOST, _stream(stream)), "gv_bc")
        return out

    def bc_multi(self, requests, stream=None) -> np.ndarray:
        """Scores of several source sets at once (gv_bc_multi): row r of the
        result is bc(requests[r]); an empty set means every vertex."""
        sets = [np.ascontiguousarray(r, dtype=np.uint32) for r in requests]
        off = np.zeros(len(sets) + 1, np.uint64)
        off[1:] = np.cumsum([len(r) for r in sets])
        flat = np.ascontiguousarray(np.concatenate(sets) if sets else np.empty(0, np.uint32), dtype=np.uint32)
        out = np.empty((len(sets), self.n), np.float32)
        _check(_lib.lib().gv_bc_multi(self._h, flat.ctypes.data if len(flat) else None, off.ctypes.data,
                                      len(sets), out.ctypes.data, GV_MEM_HOST, _stream(stream)), "gv_bc_multi")
        return out

    def bfs_sigma(self, source: int, stream=None):
        dist = np.empty(self.n, np.int32)
        sigma = np.empty(self.n, np.uint64)
        _check(_lib.lib().gv_bfs_sigma(self._h, source, dist.ctypes.data, sigma.ctypes.data, GV_MEM_HOST,
                                       _stream(stream)), "gv_bfs_sigma")
        return dist, sigma

    # -- differentiation ---------------------------------------------------
    def wpr_forward(self, alpha: float = 0.85, tol: float = 1e-7, max_iter: int = 200, stream=None):
        x = np.empty(self.n, np.float32)
        sw = C.c_int32()
        _check(_lib.lib().gv_wpr_forward(self._h, alpha, tol, max_iter, x.ctypes.data, C.byref(sw), GV_MEM_HOST,
                                         _stream(stream)), "gv_wpr_forward")
        return x, sw.value

    def wpr_backward(self, x, c, alpha: float = 0.85, tol: float = 1e-7, max_iter: int = 200, mode: int = 0,
                     stream=None):
        """(grad per entry in export order, lambda, sweeps)."""
        m = self.num_edges()
        xa = np.ascontiguousarray(x, dtype=np.float32)
        ca = np.ascontiguousarray(c, dtype=np.float32)
        grad = np.empty(max(m, 1), np.float32)
        lam = np.empty(self.n, np.float32)
        sw = C.c_int32()
        _check(_lib.lib().gv_wpr_backward(self._h, alpha, tol, max_iter, xa.ctypes.data, ca.ctypes.data, mode,
                                          grad.ctypes.data, m, lam.ctypes.data, C.byref(sw), GV_MEM_HOST,
                                          _stream(stream)), "gv_wpr_backward")
        return grad[:m], lam, sw.value

    # -- serving -----------------------------------------------------------
    def serve(self, trace, *, slots: int = 4, ppr_batch: int = 32, max_coalesce: int = 64, pace: bool = True,
              hbm_budget_bytes: int = 32 << 30, alpha: float = 0.85, epsilon: float = 1e-6, max_iter: int = 100,
              outputs: bool = False, fresh: bool = True):
        """Run a request trace through gv_serve_trace.

        trace items (arrival_s last, non-decreasing):
          ("update", ins_src, ins_dst, del_src, del_dst, arrival_s)
          ("ppr", source, arrival_s)
          ("tc", vertices, arrival_s)      incident-triangle counts of the vertices
          ("bc", sources, arrival_s)       betweenness from the given sources
        fresh=True lets a query see updates that arrived after it (never fewer
        than those before it); fresh=False gives it exactly those before it.
        Returns (results, outs): results a structured array with start_s, done_s,
        latency_ms, epoch, status, sweeps, group per request (epoch = update
        requests, in trace order, applied before the query ran); outs a list
        with each query's result (None for updates) when outputs=True."""
        kinds = {"update": _lib.GV_REQ_UPDATE, "ppr": _lib.GV_REQ_PPR, "tc": _lib.GV_REQ_TC, "bc": _lib.GV_REQ_BC}
        nreq = len(trace)
        reqs = (_lib.gv_request * max(nreq, 1))()
        srcs, dsts, qv = [], [], []
        upd_off = q_off = 0
        for i, item in enumerate(trace):
            r = reqs[i]
            r.kind = kinds[item[0]]
            r.arrival_s = float(item[-1])
            if item[0] == "update":
                ins_s, ins_d, del_s, del_d = (np.asarray(a, np.uint32) for a in item[1:5])
                r.count0, r.count1, r.offset = len(ins_s), len(del_s), upd_off
                srcs += [ins_s, del_s]
                dsts += [ins_d, del_d]
                upd_off += len(ins_s) + len(del_s)
            elif item[0] == "ppr":
                r.source = int(item[1])
            else:
                v = np.asarray(item[1], np.uint32)
                r.count0, r.offset = len(v), q_off
                qv.append(v)
                q_off += len(v)
        src = np.concatenate(srcs) if srcs else np.zeros(1, np.uint32)
        dst = np.concatenate(dsts) if dsts else np.zeros(1, np.uint32)
        qvert = np.concatenate(qv) if qv else np.zeros(1, np.uint32)
        cfg = _lib.gv_serve_config()
        L = _lib.lib()
        _check(L.gv_serve_config_init(C.byref(cfg)), "gv_serve_config_init")
        cfg.slots, cfg.ppr_batch, cfg.max_coalesce, cfg.pace = slots, ppr_batch, max_coalesce, int(pace)
        cfg.hbm_budget_bytes, cfg.alpha, cfg.epsilon, cfg.max_iter = hbm_budget_bytes, alpha, epsilon, max_iter
        cfg.fresh = int(fresh)
        res = (_lib.gv_request_result * max(nreq, 1))()
        outs_list = [None] * nreq
        po = None
        if outputs:
            ptr_ppr = (C.c_void_p * max(nreq, 1))()
            ptr_tc = (C.c_void_p * max(nreq, 1))()
            ptr_bc = (C.c_void_p * max(nreq, 1))()
            for i, item in enumerate(trace):
                if item[0] == "ppr":
                    outs_list[i] = np.zeros(self.n, np.float32)
                    ptr_ppr[i] = outs_list[i].ctypes.data
                elif item[0] == "tc":
                    outs_list[i] = np.zeros(len(item[1]), np.uint64)
                    ptr_tc[i] = outs_list[i].ctypes.data
                elif item[0] == "bc":
                    outs_list[i] = np.zeros(self.n, np.float32)
                    ptr_bc[i] = outs_list[i].ctypes.data
            po = _lib.gv_serve_outputs(C.cast(ptr_ppr, C.c_void_p), C.cast(ptr_tc, C.c_void_p),
                                       C.cast(ptr_bc, C.c_void_p))
        _check(L.gv_serve_trace(self._h, C.byref(cfg), reqs, nreq, src.ctypes.data, dst.ctypes.data,
                                qvert.ctypes.data, res, C.byref(po) if po is not None else None), "gv_serve_trace")
        dt = np.dtype([("start_s", np.float64), ("done_s", np.float64), ("latency_ms", np.float64),
                       ("epoch", np.uint32), ("status", np.uint32), ("sweeps", np.uint32), ("group", np.uint32)])
        out = np.frombuffer(bytes(res), dtype=dt, count=nreq).copy() if nreq else np.zeros(0, dt)
        return out, outs_list
