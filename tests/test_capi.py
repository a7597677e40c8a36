"""The C ABI library: it loads, exports every symbol include/aldic_b200.h
declares, and its pure-host entry points agree with the oracle.  No GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "aldic_b200.h")).read()
    return sorted(set(re.findall(r"ALDIC_API\s+[\w\s\*]*?\b(aldic_\w+)\s*\(", src)))


def test_header_lists_entry_points():
    syms = header_symbols()
    assert len(syms) >= 20
    for s in ("aldic_icgn", "aldic_subpb1", "aldic_subpb2", "aldic_int_search", "aldic_frame",
              "aldic_ba_interp2_f64", "aldic_ba_interp2_f32"):
        assert s in syms


def test_library_exports_every_header_symbol(aldic):
    L = aldic._lib.lib()
    for s in header_symbols():
        assert hasattr(L, s), s
    # the Python binding declares a signature for each of them
    assert set(header_symbols()) <= set(aldic.exported_symbols())


def test_search_dims_matches_oracle(aldic, oracle):
    L = aldic._lib.lib()
    for (W, H, w, step, s) in [(512, 512, 20, 10, 20), (2048, 2048, 32, 8, 16), (300, 200, 16, 7, 3)]:
        nx, ny = C.c_int(), C.c_int()
        gx = (C.c_int * 2)(1, W)
        gy = (C.c_int * 2)(1, H)
        sr = (C.c_int * 2)(s, s)
        assert L.aldic_search_dims(W, H, gx, gy, w, step, sr, C.byref(nx), C.byref(ny)) == 0
        assert (nx.value, ny.value) == oracle.search_dims(W, H, [1, W], [1, H], w, step, [s, s])[:2]
    bad = L.aldic_search_dims(100, 100, gx, gy, 0, 5, sr, C.byref(nx), C.byref(ny))
    assert bad == -1 and b"positive" in L.aldic_last_error()


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_have_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly(aldic):
    with pytest.raises(aldic.AldicError) as e:
        aldic.Context(0)
    assert "aldic_ctx_create" in str(e.value)


def test_null_arguments_rejected(aldic):
    L = aldic._lib.lib()
    assert L.aldic_ctx_create(0, None) == -1
    assert L.aldic_ba_interp2_f64(None, 1, 1, 1, None, None, 1, None, None) == -1
    assert b"bad arguments" in L.aldic_last_error()
