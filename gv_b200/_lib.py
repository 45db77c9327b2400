"""ctypes binding of libgv.so (the C ABI in include/*.h).

The library is loaded from this package directory only; there is no CPU
fallback, so a missing library is an ImportError.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgv.so"

GV_OK, GV_ERR_INVALID, GV_ERR_NOMEM, GV_ERR_CUDA, GV_ERR_TIMEOUT, GV_ERR_STATE, GV_ERR_UNSUPPORTED, GV_ERR_CAPACITY = range(8)
STATUS_NAMES = {0: "GV_OK", 1: "GV_ERR_INVALID", 2: "GV_ERR_NOMEM", 3: "GV_ERR_CUDA", 4: "GV_ERR_TIMEOUT",
                5: "GV_ERR_STATE", 6: "GV_ERR_UNSUPPORTED", 7: "GV_ERR_CAPACITY"}
GV_MEM_HOST, GV_MEM_DEVICE = 0, 1


class gv_config(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint32),
        ("block_size", C.c_uint32),
        ("threads_per_vertex", C.c_uint32),
        ("directed", C.c_uint32),
        ("weighted", C.c_uint32),
        ("device", C.c_int32),
        ("pool_blocks", C.c_uint64),
        ("hbm_budget_bytes", C.c_uint64),
        ("max_batch_pairs", C.c_uint64),
    ]


class gv_batch_desc(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("n_insert", C.c_uint32), ("n_delete", C.c_uint32)]


class gv_tune_result(C.Structure):
    _fields_ = [("block_size", C.c_uint32), ("threads_per_vertex", C.c_uint32), ("update_ms", C.c_float),
                ("pagerank_ms", C.c_float)]


GV_BATCH_COMPACT, GV_BATCH_GRAPH = 1, 2

GV_REQ_UPDATE, GV_REQ_PPR, GV_REQ_TC, GV_REQ_BC = range(4)


class gv_mtx_info(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("cols", C.c_uint64), ("entries", C.c_uint64), ("pattern", C.c_uint32),
                ("symmetric", C.c_uint32)]


class gv_request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("count0", C.c_uint32), ("count1", C.c_uint32), ("source", C.c_uint32),
                ("offset", C.c_uint64), ("arrival_s", C.c_double)]


class gv_request_result(C.Structure):
    _fields_ = [("start_s", C.c_double), ("done_s", C.c_double), ("latency_ms", C.c_double),
                ("epoch", C.c_uint32), ("status", C.c_uint32), ("sweeps", C.c_uint32), ("group", C.c_uint32)]


class gv_serve_config(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("ppr_batch", C.c_uint32), ("max_coalesce", C.c_uint32),
                ("pace", C.c_uint32), ("hbm_budget_bytes", C.c_uint64), ("alpha", C.c_float),
                ("epsilon", C.c_float), ("max_iter", C.c_int32), ("fresh", C.c_uint32)]


class gv_serve_outputs(C.Structure):
    _fields_ = [("ppr", C.c_void_p), ("tc", C.c_void_p), ("bc", C.c_void_p)]

P = C.c_void_p
u32, u64, i32, f32 = C.c_uint32, C.c_uint64, C.c_int32, C.c_float
pu32, pu64, pi32, pf32, pu8 = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_uint8)

# name -> (restype, argtypes); every symbol declared in include/*.h
SIGNATURES = {
    "gv_config_init": (C.c_int, [C.POINTER(gv_config), u32]),
    "gv_create": (C.c_int, [C.POINTER(gv_config), C.POINTER(P)]),
    "gv_view_create": (C.c_int, [P, C.POINTER(P)]),
    "gv_destroy": (C.c_int, [P]),
    "gv_bulk_build_csr": (C.c_int, [P, P, P, P, C.c_int, P]),
    "gv_insert_edges": (C.c_int, [P, P, P, P, u64, C.c_int, P]),
    "gv_delete_edges": (C.c_int, [P, P, P, u64, C.c_int, P]),
    "gv_compact": (C.c_int, [P, P]),
    "gv_add_vertices": (C.c_int, [P, u32, pu32, P]),
    "gv_delete_vertices": (C.c_int, [P, P, u64, u32, C.c_int, P]),
    "gv_synchronize": (C.c_int, [P, P]),
    "gv_num_vertices": (C.c_int, [P, pu32]),
    "gv_num_edges": (C.c_int, [P, pu64]),
    "gv_pool_stats": (C.c_int, [P, pu64, pu64]),
    "gv_get_config": (C.c_int, [P, C.POINTER(gv_config)]),
    "gv_degrees": (C.c_int, [P, P, C.c_int, P]),
    "gv_vertex_records": (C.c_int, [P, P]),
    "gv_export_csr": (C.c_int, [P, P, P, P, u64, C.c_int, P]),
    "gv_affected": (C.c_int, [P, P, C.c_int, P]),
    "gv_clear_affected": (C.c_int, [P, P]),
    "gv_check": (C.c_int, [P, pu64, pu32, pu32]),
    "gv_last_stat": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_double)]),
    "gv_pagerank": (C.c_int, [P, f32, f32, i32, P, pi32, C.c_int, P]),
    "gv_pagerank_dynamic": (C.c_int, [P, f32, f32, i32, P, pi32, C.c_int, P]),
    "gv_pagerank_noalloc": (C.c_int, [P, f32, f32, i32, P, pi32, P]),
    "gv_ppr": (C.c_int, [P, u32, f32, f32, i32, P, pi32, C.c_int, P]),
    "gv_tc": (C.c_int, [P, P, pu64, C.c_int, P]),
    "gv_tc_subset": (C.c_int, [P, P, u64, P, C.c_int, P]),
    "gv_update_tc": (C.c_int, [P, P, P, P, u64, P, P, u64, u32, C.POINTER(C.c_int64), P, C.c_int, P]),
    "gv_bc": (C.c_int, [P, P, u64, P, C.c_int, P]),
    "gv_bc_multi": (C.c_int, [P, P, P, u32, P, C.c_int, P]),
    "gv_bfs_sigma": (C.c_int, [P, u32, P, P, C.c_int, P]),
    "gv_wpr_forward": (C.c_int, [P, f32, f32, i32, P, pi32, C.c_int, P]),
    "gv_wpr_backward": (C.c_int, [P, f32, f32, i32, P, P, i32, P, u64, P, pi32, C.c_int, P]),
    "gv_kernel_launches": (u64, []),
    "gv_profile_enable": (C.c_int, [i32]),
    "gv_profile_reset": (C.c_int, []),
    "gv_profile_query": (C.c_int, [C.c_char_p, C.POINTER(C.c_double), pu64]),
    "gv_last_error_string": (C.c_char_p, []),
    "gv_version": (C.c_char_p, []),
    "gv_batch_run": (C.c_int, [P, C.POINTER(gv_batch_desc), u32, P, P, C.c_int, u32, P]),
    "gv_batch_run_ppr": (C.c_int, [P, C.POINTER(gv_batch_desc), u32, P, P, C.c_int, u32, P, u32, C.c_float,
                                   C.c_float, C.c_int32, P, P, P]),
    "gv_ppr_batch": (C.c_int, [P, P, u32, f32, f32, i32, P, pi32, C.c_int, P]),
    "gv_autotune": (C.c_int, [C.POINTER(gv_config), P, P, u64, C.POINTER(gv_batch_desc), u32, P, P, C.c_int,
                              C.POINTER(gv_tune_result), pu32, C.POINTER(gv_config)]),
    "gv_serve_config_init": (C.c_int, [C.POINTER(gv_serve_config)]),
    "gv_serve_trace": (C.c_int, [P, C.POINTER(gv_serve_config), C.POINTER(gv_request), u32, P, P, P,
                                 C.POINTER(gv_request_result), C.POINTER(gv_serve_outputs)]),
    "gv_mtx_parse": (C.c_int, [C.c_void_p, u64, C.c_int, C.POINTER(gv_mtx_info), P, P, P, u64, pu64, P]),
    "gv_graph_from_mtx": (C.c_int, [C.c_char_p, C.POINTER(gv_config), C.POINTER(P)]),
    "gv_snapshot_save": (C.c_int, [P, C.c_char_p]),
    "gv_snapshot_load": (C.c_int, [C.c_char_p, C.POINTER(gv_config), C.POINTER(P)]),
    "gv_gen_rmat": (C.c_int, [u32, u64, u64, u64, P, P, C.c_int, P]),
    "gv_gen_uniform": (C.c_int, [u32, u64, u64, P, P, C.c_int, P]),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m gv_b200.build` "
                              "(libgv has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
