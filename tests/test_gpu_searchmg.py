"""Multigrid search on the GPU (aldic_int_search_mg through funIntegerSearchMg)
against the oracle's restatement of funIntegerSearchMg.m: the data-dependent
node grid, the level-1 (whole ROI) shift, the region count and failures, and
u, v, cc.max and the q-factors after gridfit.  Cases: a square ROI with a
displacement larger than the subset; a 4:1 ROI (x-only splits, repeated
regions) with a constant patch whose regions raise in normxcorr2 (NaN, Phi
0, separate gridfit data sets); 16-bit images."""
import numpy as np
import pytest

from oracle import searchmg as S

pytestmark = pytest.mark.gpu


def _check(aldic, f, g, gridx, gridy, w, step):
    ro = S.int_search_mg(f, g, gridx, gridy, w, step)
    info = {}
    x, y, u, v, cc = aldic.funIntegerSearchMg(f, g, gridx, gridy, w, step, step, info=info)
    np.testing.assert_array_equal(x, ro["x"])
    np.testing.assert_array_equal(y, ro["y"])
    u1, v1 = ro["regions"]["level1"]
    # level 1 by FP64 FFT on the GPU, exact sums in the oracle: the 1e-3-rounded
    # peak agrees
    assert (info["level1_u"], info["level1_v"]) == (u1, v1)
    assert info["regions"] == len(ro["regions"]["regions"])
    assert info["failed"] == ro["regions"]["failed"]
    for got, ref in ((u, ro["u"]), (v, ro["v"]), (cc["max"], ro["ccmax"])):
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-8)
    np.testing.assert_allclose(cc["qfactors"][:, 0], ro["q1"].T.reshape(-1), rtol=0, atol=1e-8)
    np.testing.assert_allclose(cc["qfactors"][:, 1], ro["q2"].T.reshape(-1), rtol=0, atol=1e-8)
    return ro, info, (x, y, u, v)


def test_mg_large_shift_matches_oracle(aldic, synth):
    W = H = 192
    f = synth.speckle(W, H, 1100, 7)
    fld = lambda X, Y: (23.3 + 0.01 * X, -17.6 + 0.5 * np.sin(2 * np.pi * Y / 150))
    g = synth.warp(f, fld, 2.0, 7)
    ro, info, (x, y, u, v) = _check(aldic, f, g, [1, W], [1, H], 16, 8)
    ut, vt = fld(x, y)
    assert np.median(np.abs(u - ut)) < 0.1 and np.median(np.abs(v - vt)) < 0.1
    assert info["levels"] >= 4 and info["failed"] == 0


def test_mg_wide_roi_with_flat_patch(aldic, synth):
    W, H = 320, 96
    f = synth.speckle(W, H, 1000, 8)
    f[30:70, 120:170] = 60                    # constant: normxcorr2 raises there
    fld = lambda X, Y: (3.4 + 0.002 * X, -2.2 + 0 * Y)
    g = synth.warp(f, fld, 2.0, 8)
    ro, info, _ = _check(aldic, f, g, [1, W], [1, H], 16, 8)
    assert info["failed"] > 0
    # failed regions carry NaN u (dropped by gridfit) but Phi = 0 (kept)
    R = ro["regions"]
    assert np.isnan(R["u"]).sum() == info["failed"] and (R["phi"][np.isnan(R["u"])] == 0).all()


def test_mg_uint16(aldic, synth):
    W = H = 160
    f = synth.speckle(W, H, 800, 9, dtype=np.uint16, scale=257.0)
    g = synth.warp(f, lambda X, Y: (-11.6 + 0 * X, 8.3 + 0.005 * Y), 2.0 * 257, 9)
    _check(aldic, f, g, [1, W], [1, H], 20, 10)


def test_mg_rejects_bad_arguments(aldic, synth):
    f = synth.speckle(64, 64, 100, 1)
    with pytest.raises(aldic.AldicError):
        aldic.funIntegerSearchMg(f, f, [1, 64], [1, 64], 0, 8, 8)


def test_frame_with_multigrid_init(aldic, synth):
    """main_ALDIC.m with the multigrid search (IntegerSearch.m:117-120): the
    search decides the node grid, MeshSetUp/Init follow, the ADMM frame runs
    on it; identical to a frame given the same U0 on that explicit grid; a
    later frame (previous U) keeps the grid."""
    W = H = 256
    f = synth.speckle(W, H, 2000, 11)
    fld = lambda X, Y: (30.2 + 0.004 * X, -21.7 + 0.6 * np.sin(2 * np.pi * Y / 200))
    g = synth.warp(f, fld, 2.0, 11)
    x, y, u, v, _ = aldic.funIntegerSearchMg(f, g, [1, W], [1, H], 20, 10, 10)
    ny, nx = u.shape
    al = aldic.ALDIC(20, 10, 0, tol=1e-3, n_admm=2, precision=aldic.FP64)
    al.set_images(f, g)
    r = al.frame(init=aldic.INIT_SEARCH_MG)
    assert (r["M"], r["N"]) == (nx, ny)
    assert r["node_grid"] == (x[0, 0], y[0, 0], nx, ny)
    np.testing.assert_array_equal(r["x0"], x.reshape(-1))
    np.testing.assert_array_equal(r["y0"], y.reshape(-1))
    assert r["stats"]["t_search_mg_ms"] > 0
    # the same frame from the same U0 on the explicit grid
    U0 = np.empty(2 * nx * ny)
    U0[0::2], U0[1::2] = u.reshape(-1), v.reshape(-1)
    al.set_init(U0)
    r2 = al.frame(init=aldic.INIT_GIVEN)
    for k in ("U", "F", "iters"):
        np.testing.assert_array_equal(r2[k], r[k])
    # accuracy against the field at the nodes (displacements > the subset size)
    ut, vt = fld(r["x0"], r["y0"])
    e = np.r_[r["U"][0::2] - ut, r["U"][1::2] - vt]
    assert np.median(np.abs(e)) < 0.02 and np.sqrt(np.mean(e ** 2)) < 0.06   # border nodes worst
    # the next frame starts from this one's U on the same grid
    r3 = al.frame(init=aldic.INIT_PREV)
    assert (r3["M"], r3["N"]) == (nx, ny)
    np.testing.assert_array_equal(r3["x0"], r["x0"])
    assert np.abs(r3["U"] - r["U"]).max() < 0.05     # same images, restarted from U
