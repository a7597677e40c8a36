"""ctypes binding of libaldic_b200.so (the C ABI of include/aldic_b200.h).

The library is built in-tree (build.py).  Importing this module never falls
back to anything else: a missing or unloadable library raises at once.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaldic_b200.so")

P = C.c_void_p
I32 = C.c_int
I64 = C.c_int64
D = C.c_double

_SIGS = {
    "aldic_version": ([], I32),
    "aldic_last_error": ([], C.c_char_p),
    "aldic_ba_interp2_f64": ([P, I64, I64, I64, P, P, I64, P, P], I32),
    "aldic_ba_interp2_f32": ([P, I64, I64, I64, P, P, I64, P, P], I32),
    "aldic_ctx_create": ([I32, P], I32),
    "aldic_ctx_destroy": ([P], I32),
    "aldic_ctx_set_stream": ([P, P], I32),
    "aldic_set_ref": ([P, P, I32, I32, I32, P, P], I32),
    "aldic_set_def": ([P, P, I32], I32),
    "aldic_set_fields": ([P, P, P, P, P, I32, I32], I32),
    "aldic_normalize": ([P, P, I32, I32, I32, P, P, P], I32),
    "aldic_gradient": ([P, P, I32, I32, P, P, P], I32),
    "aldic_get_images": ([P, P, P, P, P, P], I32),
    "aldic_search_dims": ([I32, I32, P, P, I32, I32, P, P, P], I32),
    "aldic_int_search": ([P, P, P, I32, I32, P, P, P, P, P, P, P], I32),
    "aldic_int_search_mg": ([P, P, P, I32, I32, P, P, I64, P, P, P, P, P, P, P], I32),
    "aldic_icgn": ([P, P, I64, P, P, I32, D, I32, P, P, P, P], I32),
    "aldic_localicgn_post": ([P, I32, I32, P, P, P, P], I32),
    "aldic_subpb1": ([P, P, I64, P, P, P, P, P, I32, D, D, I32, P, P], I32),
    "aldic_subpb1_post": ([P, I32, I32, P, P, P], I32),
    "aldic_subpb2": ([P, I32, I32, D, D, D, P, P, P, P, P], I32),
    "aldic_subpb2_noalloc": ([I32, I32, D, D, D, P, P, P, P, P, P], I32),
    "aldic_nodal_strain": ([P, I32, I32, D, P, P], I32),
    "aldic_gridfit_springs": ([P, I32, I32, I32, P, P], I32),
    "aldic_inpaint_springs": ([P, I32, I32, I32, P], I32),
    "aldic_smooth": ([P, I32, I32, I32, P], I32),
    "aldic_frame_dims": ([P, P, P, P], I32),
    "aldic_frame": ([P, P, P, P, P, P, P, P], I32),
    "aldic_set_init": ([P, P, I64], I32),
    "aldic_qt_mesh_generate": ([I32, P, I32, P, P, I32, I32, D, I32, P], I32),
    "aldic_qt_mesh_create": ([I32, P, I32, P, I32, P, P], I32),
    "aldic_qt_mesh_info": ([P, P, P, P], I32),
    "aldic_qt_mesh_get": ([P, P, P, P], I32),
    "aldic_qt_mesh_destroy": ([P], I32),
    "aldic_qt_subpb2": ([P, P, D, D, P, P, P], I32),
    "aldic_qt_nodal_strain": ([P, P, P, P], I32),
    "aldic_qt_fill": ([P, P, I32, P, P], I32),
    "aldic_icgn_flags": ([P, I64, P, D, P, P], I32),
    "aldic_subpb2_fd": ([P, I32, I32, D, D, D, P, P, P, P, P], I32),
    "aldic_fd_strain": ([P, I32, I32, D, P, P], I32),
    "aldic_compute_strain": ([P, I32, I32, D, I32, I32, I32, P, P, P, P], I32),
    "aldic_fdm_basis": ([I32, I32, D, P, P], I32),
    "aldic_set_stats": ([P, P], I32),
    "aldic_qt_frame": ([P, P, P, P], I32),
    "aldic_qt_frame_get": ([P, P, P, P, P, P, P], I32),
    "aldic_set_init_gated": ([P, P, P, P, D, I64], I32),
    "aldic_icgn_autotune": ([I32], I32),
    "aldic_icgn_shape": ([I32, I32, I32, C.c_longlong, P, P, P, P], I32),
    "aldic_gemm_bf16": ([P, P, P, P, I32, I32], I32),
    "aldic_cnn_create": ([I32, C.c_uint64, P], I32),
    "aldic_cnn_destroy": ([P], I32),
    "aldic_cnn_num_params": ([], I64),
    "aldic_cnn_get_params": ([P, P], I32),
    "aldic_cnn_set_params": ([P, P], I32),
    "aldic_cnn_train_step": ([P, P, I32, P, I32, C.c_float, P, P, P, P], I32),
    "aldic_cnn_predict": ([P, P, I32, I32, P, P], I32),
    "aldic_cnn_patches": ([P, P, I64, I32, P], I32),
    "aldic_cnn_to_init": ([P, P, I64, P, P, P], I32),
}


class FrameParams(C.Structure):
    _fields_ = [("winsize", I32), ("step", I32), ("search", I32 * 2), ("gridx", I32 * 2),
                ("gridy", I32 * 2), ("tol", D), ("mu", D), ("beta", D), ("n_admm", I32),
                ("tol2", D), ("precision", I32), ("smooth", I32), ("use_graph", I32),
                ("init", I32), ("subpb2_fd", I32), ("node_grid", D * 4)]


class GemmOperand(C.Structure):
    _fields_ = [("p", P), ("ld", I64), ("mode", I32), ("rows", I64), ("kdim", I64),
                ("Hin", I32), ("Win", I32), ("C", I32), ("ps", I32), ("bstride", I64)]


class GemmOutput(C.Structure):
    _fields_ = [("p", P), ("ld", I64), ("mode", I32), ("fp32", I32), ("bias", P), ("relu", I32),
                ("mask", P), ("Hin", I32), ("Win", I32), ("C", I32), ("ps", I32), ("M", I64),
                ("N", I64), ("split_stride", I64), ("scale", C.c_float), ("bstride", I64)]


class FrameStats(C.Structure):
    _fields_ = [("M", I32), ("N", I32), ("admm_steps", I32), ("bad_icgn", I32),
                ("converged_icgn", I32), ("beta", D), ("update_y", D * 16),
                ("update_y2", D * 16), ("mean_iters_icgn", D), ("kernel_launches", I32),
                ("t_stage_ms", D * 8), ("max_pcg_iters", I32), ("node_grid", D * 4),
                ("t_search_mg_ms", D), ("gated_init", I32)]


class QtFrameParams(C.Structure):
    _fields_ = [("winsize", I32), ("step", I32), ("search", I32), ("gridx", I32 * 2),
                ("gridy", I32 * 2), ("tol", D), ("mu", D), ("tol2", D), ("n_admm", I32),
                ("min_size", I32), ("precision", I32), ("subsets", I32)]


class QtFrameStats(C.Structure):
    _fields_ = [("n", I32), ("ne", I32), ("ndir", I32), ("bad_icgn", I32), ("admm_steps", I32),
                ("mesh_reused", I32), ("beta", D), ("update_y", D * 16), ("update_y2", D * 16),
                ("t_ms", D * 6)]


class AldicError(RuntimeError):
    """A non-zero status from the C ABI (message from aldic_last_error)."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python 2d_aldic_b200/build.py` "
                "(the CUDA path has no fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def call(name: str, *args) -> int:
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        msg = lib().aldic_last_error()
        raise AldicError(name, rc, msg.decode() if msg else "")
    return rc
