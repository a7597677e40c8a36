"""The IC-GN launch-shape autotuner (k_icgn.cu): every candidate shape runs
the same per-subset code, so a tuned launch (which runs each shape twice on
the call's own data and keeps the last outputs) returns exactly what the
default shape returns, for LocalICGN and Subpb1, FP32 and FP64; the chosen
shape and the trial times are reported."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_tuned_shapes_give_identical_results(aldic, oracle, synth, prec):
    wl = synth.workload("plain512")
    f, g = wl.images()
    H, W = f.shape
    gn, mg, _ = oracle.normalize(g)
    x, y, u, v, _, _ = oracle.int_search(f, g, mg, [1, W], [1, H], wl.winsize, wl.step,
                                         [wl.search, wl.search])
    # the grid twice over: the tuner runs on launches of 2048 subsets or more
    coords = np.tile(np.stack([x.ravel(), y.ravel()], 1), (2, 1))
    n = len(coords)
    assert n >= 2048
    U0 = np.empty(2 * n)
    U0[0::2], U0[1::2] = np.tile(u.ravel(), 2), np.tile(v.ravel(), 2)
    p = aldic.FP64 if prec == "fp64" else aldic.FP32
    lib = aldic._lib.lib()
    ctx = aldic.Context(0)
    try:
        ctx.set_ref(f)
        ctx.set_def(g)
        lib.aldic_icgn_autotune(0)
        U_d, F_d, it_d, H_d = aldic.local_icgn(ctx, coords, U0, wl.winsize, wl.tol, p)
        lib.aldic_icgn_autotune(1)
        U_t, F_t, it_t, H_t = aldic.local_icgn(ctx, coords, U0, wl.winsize, wl.tol, p)
        for a, b in ((U_d, U_t), (F_d, F_t), (it_d, it_t), (H_d, H_t)):
            np.testing.assert_array_equal(a, b)
        nw, mb, cnt = C.c_int(), C.c_int(), C.c_int()
        ms = (C.c_float * 8)()
        assert lib.aldic_icgn_shape(int(p), 0, wl.winsize, C.c_longlong(n), C.byref(nw), C.byref(mb),
                                    ms, C.byref(cnt)) == 0
        assert cnt.value >= 2 and nw.value in (4, 8, 16)
        assert all(ms[k] > 0 for k in range(cnt.value))
        # Subpb1 (funICGN_Subpb1) from the IC-GN result: default shape vs tuned
        vd = 0.01 * np.random.default_rng(2).standard_normal(2 * n)
        H21 = np.ascontiguousarray(H_d.T)          # n x 21 column-major
        cf = np.ascontiguousarray(coords.T)
        ptr = lambda a: C.c_void_p(a.ctypes.data)

        def sub():
            Uo = np.empty(2 * n)
            it = np.empty(n, np.int32)
            aldic._lib.call("aldic_subpb1", ctx.h, ptr(cf), n, ptr(U_d), ptr(F_d), ptr(vd),
                            ptr(H21), None, wl.winsize, 1e-3, wl.tol, int(p), ptr(Uo), ptr(it))
            return Uo, it

        lib.aldic_icgn_autotune(0)
        a = sub()
        lib.aldic_icgn_autotune(1)
        b = sub()
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        assert lib.aldic_icgn_shape(int(p), 1, wl.winsize, C.c_longlong(n), C.byref(nw), C.byref(mb),
                                    ms, C.byref(cnt)) == 0
    finally:
        ctx.close()
