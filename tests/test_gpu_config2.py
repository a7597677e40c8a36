"""The headline workload against the FP64 oracle, exactly as bench.py runs it:
2048 x 2048 8-bit speckle (130k dots, seed 1), u = 2 sin(2 pi y/256),
v = 1.5 cos(2 pi x/256), noise 2; subset 32, step 8 (59 049 subsets), search
+-16 px, IC-GN tol 1e-2, 3 ADMM iterations.

Tolerances (the path's specification): integer-search peaks bit-exact; the
FP64 frame within 1e-4 px of the oracle frame (U and F after the same ADMM
iteration count); the FP32-sampling frame within 0.01 px RMS; FP32 IC-GN
within 1e-3 px (U) and 1e-5 (F) on every subset converged in both runs with
the same iteration count, and within one stopping-test step where the counts
differ (see test_gpu_parity.check_icgn_converged).
"""
import numpy as np
import pytest

from test_gpu_parity import check_icgn_converged

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2(synth, oracle):
    wl = synth.workload("uniform2048")
    f, g = wl.images()
    ro = oracle.frame(f, g, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=wl.n_admm)
    return wl, f, g, ro


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_config2_frame_matches_oracle(aldic, c2, prec):
    wl, f, g, ro = c2
    al = aldic.ALDIC(wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=wl.n_admm,
                     precision=aldic.FP64 if prec == "fp64" else aldic.FP32)
    al.set_images(f, g)
    r = al.frame()
    assert r["M"] * r["N"] == 59049
    np.testing.assert_array_equal(r["x0"], ro["x0"])
    np.testing.assert_array_equal(r["y0"], ro["y0"])
    # LocalICGN's -1 subsets (688 here: more than 10 % zero-gradient pixels
    # grow the window to an odd size, whose bounds are not integral) and 102
    it, ito = np.asarray(r["iters"]).ravel(), np.asarray(ro["iters_icgn"]).ravel()
    for code in (-1, 102):
        np.testing.assert_array_equal(it == code, ito == code)
    dU = r["U"] - ro["U"]
    dF = r["F"] - ro["F"]
    rms = float(np.sqrt(np.mean(dU ** 2)))
    print(f"config 2 {prec}: max |dU| {np.abs(dU).max():.3g} px, RMS {rms:.3g} px, "
          f"max |dF| {np.abs(dF).max():.3g}, beta {r['stats']['beta']:.6g} vs {ro['beta']:.6g}")
    # the beta sweep (its six systems solved from the right-hand side's two
    # parts, the errors in one pass) selects the oracle's beta
    assert r["stats"]["beta"] == pytest.approx(ro["beta"], rel=1e-6)
    if prec == "fp64":
        assert np.abs(dU).max() < 1e-4 and np.abs(dF).max() < 1e-4
    else:
        assert rms < 0.01


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_config2_icgn_all_converged_subsets(aldic, oracle, c2, prec):
    """LocalICGN (funICGN per subset) from the integer-search start, every
    subset of the bench geometry."""
    wl, f, g, _ = c2
    H, W = f.shape
    fn, _, _ = oracle.normalize(f)
    gn, mg, _ = oracle.normalize(g)
    dx, dy = oracle.gradient(fn)
    x, y, u, v, _, _ = oracle.int_search(f, g, mg, [1, W], [1, H], wl.winsize, wl.step,
                                         [wl.search, wl.search])
    xs, ys, us, vs, _ = aldic.funIntegerSearch(f, g, wl.search, [1, W], [1, H], wl.winsize, wl.step,
                                               0, qfactors=False)
    for a, b in ((xs, x), (ys, y), (us, u), (vs, v)):
        np.testing.assert_array_equal(a, b)          # integer search bit-exact
    coords = np.stack([x.ravel(), y.ravel()], 1)
    U0 = np.empty(2 * x.size)
    U0[0::2], U0[1::2] = u.ravel(), v.ravel()
    ctx = aldic.Context(0)
    try:
        ctx.set_ref(f)
        ctx.set_def(g)
        U, F, it, _ = aldic.local_icgn(ctx, coords, U0, wl.winsize, wl.tol,
                                       aldic.FP64 if prec == "fp64" else aldic.FP32)
    finally:
        ctx.close()
    Uo, Fo, ito, _ = oracle.icgn_batch(fn, gn, dx, dy, coords, U0, wl.winsize, wl.tol)
    check_icgn_converged(U, F, it, Uo, Fo, ito, prec, "uniform2048")


def test_config2_split_icgn_equals_one_launch(aldic, c2):
    """The FP32 frame runs LocalICGN as a setup launch and an iteration launch
    that share a per-subset record (k_icgn.cu MODE_SETUP / MODE_ITER); the
    C ABI's aldic_icgn runs it in one launch.  Same arithmetic, so the same
    status and iteration count on every subset of the headline frame."""
    wl, f, g, _ = c2
    H, W = f.shape
    al = aldic.ALDIC(wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=0, precision=aldic.FP32)
    al.set_images(f, g)
    r = al.frame()
    xs, ys, us, vs, _ = aldic.funIntegerSearch(f, g, wl.search, [1, W], [1, H], wl.winsize, wl.step,
                                               0, qfactors=False)
    coords = np.stack([xs.ravel(), ys.ravel()], 1)
    U0 = np.empty(2 * xs.size)
    U0[0::2], U0[1::2] = us.ravel(), vs.ravel()
    ctx = aldic.Context(0)
    try:
        ctx.set_ref(f)
        ctx.set_def(g)
        _, _, it, _ = aldic.local_icgn(ctx, coords, U0, wl.winsize, wl.tol, aldic.FP32)
    finally:
        ctx.close()
    np.testing.assert_array_equal(np.asarray(r["iters"]).ravel(), it)
