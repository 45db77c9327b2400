"""CPU tests of the boundary: libgv loads and exports every entry point that
include/*.h declares; host-side argument validation needs no GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
DECL = re.compile(r"^\s*(?:gv_status|uint64_t|const\s+char\s*\*)\s*\**\s*(gv_\w+)\s*\(", re.M)


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names.update(DECL.findall(h.read_text()))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    for must in ("gv_create", "gv_insert_edges", "gv_delete_edges", "gv_compact", "gv_pagerank", "gv_tc", "gv_bc",
                 "gv_wpr_forward", "gv_wpr_backward"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from gv_b200 import _lib
    L = C.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    from gv_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_version_and_launch_counter():
    import gv_b200
    assert "sm_100a" in gv_b200.version()
    assert gv_b200.kernel_launches() >= 0


def test_config_validation_without_gpu():
    import gv_b200
    from gv_b200 import _lib
    L = _lib.lib()
    cfg = _lib.gv_config()
    assert L.gv_config_init(C.byref(cfg), 100) == 0
    assert cfg.block_size == 128 and cfg.threads_per_vertex == 8
    h = C.c_void_p()
    cfg.block_size = 48
    assert L.gv_create(C.byref(cfg), C.byref(h)) == _lib.GV_ERR_INVALID
    cfg.block_size = 128
    cfg.threads_per_vertex = 6
    assert L.gv_create(C.byref(cfg), C.byref(h)) == _lib.GV_ERR_INVALID
    assert L.gv_create(None, C.byref(h)) == _lib.GV_ERR_INVALID


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import gv_b200
    with pytest.raises(gv_b200.GvError) as e:
        gv_b200.GraphVine(64)
    assert "no CUDA device" in str(e.value) or "GV_ERR_CUDA" in str(e.value)


def test_serve_config_defaults_and_null_graph():
    from gv_b200 import _lib
    L = _lib.lib()
    cfg = _lib.gv_serve_config()
    assert L.gv_serve_config_init(C.byref(cfg)) == 0
    assert cfg.slots >= 1 and 1 <= cfg.ppr_batch <= 32 and cfg.pace == 1
    res = (_lib.gv_request_result * 1)()
    reqs = (_lib.gv_request * 1)()
    assert L.gv_serve_trace(None, C.byref(cfg), reqs, 1, None, None, None, res, None) == _lib.GV_ERR_INVALID
    assert L.gv_view_create(None, None) == _lib.GV_ERR_INVALID


def test_mtx_header_parse_without_gpu():
    from gv_b200 import _lib
    L = _lib.lib()
    info = _lib.gv_mtx_info()
    cnt = C.c_uint64()
    text = b"%%MatrixMarket matrix coordinate pattern symmetric\n% a comment\n\n 5 6 3\n1 2\n2 3\n3 1\n"
    buf = C.create_string_buffer(text, len(text))
    assert L.gv_mtx_parse(buf, len(text), 0, C.byref(info), None, None, None, 0, C.byref(cnt), None) == 0
    assert (info.rows, info.cols, info.entries, info.pattern, info.symmetric) == (5, 6, 3, 1, 1)
    bad = b"%%MatrixMarket matrix coordinate real general\nnot a size line\n"
    buf = C.create_string_buffer(bad, len(bad))
    assert L.gv_mtx_parse(buf, len(bad), 0, C.byref(info), None, None, None, 0, C.byref(cnt), None) == _lib.GV_ERR_INVALID


def test_library_leaves_none_of_its_own_symbols_undefined():
    """Every gv:: function the library calls is defined in it (a missing one
    would only show when the library is loaded with immediate binding)."""
    import os
    import subprocess
    from gv_b200 import _lib
    out = subprocess.run(["nm", "-D", "--undefined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    own = [ln for ln in out.splitlines() if "_ZN2gv" in ln]
    assert not own, own
    C.CDLL(str(_lib.LIB_PATH), mode=os.RTLD_NOW)

