"""CPU oracle for the GraphVine hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may import this package, as the checker or the timed CPU baseline.  The
product (gv_b200 / libgv) never calls it.  See oracle/gv_oracle.h for the
semantics and how the oracle is pinned.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_P = C.c_void_p
_SIG = {
    "or_create": (_P, [C.c_uint32, C.c_int, C.c_int]),
    "or_destroy": (None, [_P]),
    "or_set_threads": (C.c_int, [C.c_int]),
    "or_insert": (C.c_int, [_P, _P, _P, _P, C.c_uint64]),
    "or_insert_directed": (C.c_int, [_P, _P, _P, _P, C.c_uint64]),
    "or_delete": (C.c_int, [_P, _P, _P, C.c_uint64]),
    "or_num_edges": (C.c_uint64, [_P]),
    "or_export": (None, [_P, _P, _P, _P]),
    "or_pagerank": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _P, C.c_int, _P]),
    "or_ppr": (C.c_int, [_P, C.c_uint32, C.c_double, C.c_double, C.c_int, C.c_int, _P]),
    "or_tc": (C.c_uint64, [_P, _P]),
    "or_tc_incident": (None, [_P, _P, C.c_uint64, _P]),
    "or_bc": (None, [_P, _P, C.c_uint64, _P]),
    "or_bfs_sigma": (None, [_P, C.c_uint32, _P, _P]),
    "or_wpr_forward": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _P]),
    "or_wpr_adjoint": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _P, _P]),
    "or_wpr_gradient": (None, [_P, C.c_double, _P, _P, _P, C.c_int, _P]),
    "or_wpr_objective": (C.c_double, [_P, C.c_double, C.c_double, C.c_int, _P, C.c_uint32, C.c_uint32, C.c_double]),
    "or_wpr_fd": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _P, _P, _P, C.c_uint32, C.c_double, _P]),
    "or_rmat_pairs": (None, [C.c_uint32, C.c_uint64, C.c_uint64, _P, _P]),
    "or_uniform_pairs": (None, [C.c_uint32, C.c_uint64, C.c_uint64, _P, _P]),
}
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from . import build
            build.build()
        L = C.CDLL(str(LIB_PATH))
        for k, (r, a) in _SIG.items():
            getattr(L, k).restype = r
            getattr(L, k).argtypes = a
        _lib = L
    return _lib


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def set_threads(n: int) -> int:
    return lib().or_set_threads(n)


def rmat_pairs(scale: int, num_pairs: int, seed: int):
    s = np.empty(num_pairs, np.uint32)
    d = np.empty(num_pairs, np.uint32)
    lib().or_rmat_pairs(scale, num_pairs, seed, s.ctypes.data, d.ctypes.data)
    return s, d


def uniform_pairs(n: int, num_pairs: int, seed: int):
    """Seeded uniform pairs u != v (the generator libgv's gen_uniform uses)."""
    s = np.empty(num_pairs, np.uint32)
    d = np.empty(num_pairs, np.uint32)
    lib().or_uniform_pairs(n, num_pairs, seed, s.ctypes.data, d.ctypes.data)
    return s, d


class OracleGraph:
    def __init__(self, n: int, directed: bool = False, weighted: bool = False):
        self.n, self.directed, self.weighted = n, directed, weighted
        self._h = lib().or_create(n, int(directed), int(weighted))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_destroy(self._h)
            self._h = None

    def insert(self, src, dst, w=None, directed_entries: bool = False) -> None:
        s, d = _u32(src), _u32(dst)
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        f = lib().or_insert_directed if directed_entries else lib().or_insert
        if f(self._h, s.ctypes.data, d.ctypes.data, None if wa is None else wa.ctypes.data, len(s)) != 0:
            raise ValueError("vertex id out of range")

    def delete(self, src, dst) -> None:
        s, d = _u32(src), _u32(dst)
        if lib().or_delete(self._h, s.ctypes.data, d.ctypes.data, len(s)) != 0:
            raise ValueError("vertex id out of range")

    def num_edges(self) -> int:
        return int(lib().or_num_edges(self._h))

    def export(self):
        m = self.num_edges()
        off = np.empty(self.n + 1, np.uint64)
        dst = np.empty(max(m, 1), np.uint32)
        w = np.empty(max(m, 1), np.float32)
        lib().or_export(self._h, off.ctypes.data, dst.ctypes.data, w.ctypes.data)
        return off, dst[:m], w[:m]

    def pagerank(self, alpha=0.85, epsilon=1e-6, max_iter=100, x_init=None, fixed_sweeps=0):
        x = np.empty(self.n, np.float64)
        xi = None if x_init is None else np.ascontiguousarray(x_init, dtype=np.float64)
        sw = lib().or_pagerank(self._h, alpha, epsilon, max_iter, None if xi is None else xi.ctypes.data,
                               fixed_sweeps, x.ctypes.data)
        return x, sw

    def ppr(self, source, alpha=0.85, epsilon=1e-6, max_iter=100, fixed_sweeps=0):
        x = np.empty(self.n, np.float64)
        sw = lib().or_ppr(self._h, source, alpha, epsilon, max_iter, fixed_sweeps, x.ctypes.data)
        return x, sw

    def tc(self, per_vertex: bool = True):
        """(per-vertex counts or None, total); per_vertex=False counts the total only."""
        pv = np.empty(self.n, np.uint64) if per_vertex else None
        tot = lib().or_tc(self._h, pv.ctypes.data if per_vertex else None)
        return pv, int(tot)

    def tc_incident(self, subset):
        s = _u32(subset)
        out = np.empty(len(s), np.uint64)
        lib().or_tc_incident(self._h, s.ctypes.data, len(s), out.ctypes.data)
        return out

    def bc(self, sources=None):
        out = np.empty(self.n, np.float64)
        if sources is None:
            lib().or_bc(self._h, None, 0, out.ctypes.data)
        else:
            s = _u32(sources)
            lib().or_bc(self._h, s.ctypes.data, len(s), out.ctypes.data)
        return out

    def bfs_sigma(self, source):
        dist = np.empty(self.n, np.int32)
        sigma = np.empty(self.n, np.uint64)
        lib().or_bfs_sigma(self._h, source, dist.ctypes.data, sigma.ctypes.data)
        return dist, sigma

    def wpr_forward(self, alpha=0.85, tol=1e-14, max_iter=1000):
        x = np.empty(self.n, np.float64)
        sw = lib().or_wpr_forward(self._h, alpha, tol, max_iter, x.ctypes.data)
        return x, sw

    def wpr_adjoint(self, c, alpha=0.85, tol=1e-14, max_iter=1000):
        ca = np.ascontiguousarray(c, dtype=np.float64)
        lam = np.empty(self.n, np.float64)
        sw = lib().or_wpr_adjoint(self._h, alpha, tol, max_iter, ca.ctypes.data, lam.ctypes.data)
        return lam, sw

    def wpr_gradient(self, x, lam, c, alpha=0.85, mode=0):
        g = np.empty(max(self.num_edges(), 1), np.float64)
        xa, la, ca = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, lam, c))
        lib().or_wpr_gradient(self._h, alpha, xa.ctypes.data, la.ctypes.data, ca.ctypes.data, mode, g.ctypes.data)
        return g[: self.num_edges()]

    def wpr_fd(self, c, eu, ev, h=1e-6, alpha=0.85, tol=1e-15, max_iter=2000):
        """fp64 central differences of sum c_i x_i w.r.t. the raw weights of entries (eu[i], ev[i])."""
        ca = np.ascontiguousarray(c, dtype=np.float64)
        u, v = _u32(eu), _u32(ev)
        out = np.empty(len(u), np.float64)
        lib().or_wpr_fd(self._h, alpha, tol, max_iter, ca.ctypes.data, u.ctypes.data, v.ctypes.data, len(u), h,
                        out.ctypes.data)
        return out

    def wpr_objective(self, c, u, v, delta, alpha=0.85, tol=1e-15, max_iter=2000):
        ca = np.ascontiguousarray(c, dtype=np.float64)
        return lib().or_wpr_objective(self._h, alpha, tol, max_iter, ca.ctypes.data, u, v, delta)
