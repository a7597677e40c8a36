"""The oracle's restatement of the multigrid search (funIntegerSearchMg.m):
a displacement much larger than a subset is recovered on the node grid, the
level recursion follows the reference's split rule, and gridfit reproduces
an affine field exactly.  CPU only."""
import math

import numpy as np
import pytest

from oracle import searchmg as S


@pytest.fixture(scope="module")
def pair(synth):
    W = H = 192
    f = synth.speckle(W, H, 1100, 7)
    fld = lambda X, Y: (23.3 + 0.01 * X, -17.6 + 0.5 * np.sin(2 * np.pi * Y / 150))
    return f, synth.warp(f, fld, 2.0, 7), fld


def test_large_shift_recovered(pair):
    f, g, fld = pair
    r = S.int_search_mg(f, g, [1, 192], [1, 192], 16, 8)
    ut, vt = fld(r["x"], r["y"])
    assert np.median(np.abs(r["u"] - ut)) < 0.1 and np.median(np.abs(r["v"] - vt)) < 0.1
    assert np.abs(r["u"] - ut).max() < 0.5 and np.abs(r["v"] - vt).max() < 0.5
    # the whole-ROI level finds the mean shift to within a pixel
    u1, v1 = r["regions"]["level1"]
    assert abs(u1 - 24.2) < 1.5 and abs(v1 + 17.6) < 1.5
    # borders follow the displacement of the outermost regions
    assert r["xlist"][0] == math.ceil(1 + 1.25 * 16 + r["regions"]["u"][np.argmin(
        [0.5 * (q[0][0] + q[0][1]) for q in r["regions"]["regions"]])])
    assert np.nanmin(r["q1"]) > -0.5 and np.nanmax(r["q1"]) < 1.5


def test_split_rule_wide_roi(synth):
    """A 4:1 ROI is split in x only while its nominal aspect ratio exceeds 2;
    a region is halved only while wider than the subset (in "both" mode, in
    both directions), otherwise it is repeated (funIntegerSearchMg.m:58-147)."""
    W, H = 320, 96
    f = synth.speckle(W, H, 1000, 8)
    g = synth.warp(f, lambda X, Y: (3.0 + 0 * X, -2.0 + 0 * Y), 2.0, 8)
    R = S.regions(f, g, [1, W], [1, H], 16, float(g.mean()))
    from collections import Counter
    reps = Counter((tuple(q[0]), tuple(q[1])) for q in R["regions"])
    xs = {k[0] for k in reps}
    ys = {k[1] for k in reps}
    # ROI 294 x 70: x, x, both, both (18 x 16 regions stop splitting: 16 is not
    # wider than the subset), last level repeats each of them 4 times
    assert len(xs) == 16 and len(reps) == len(R["regions"]) // 4
    assert set(reps.values()) == {4}
    assert all(b - a <= 18 for a, b in xs) and all(b - a <= 16 for a, b in ys)
    assert np.nanmax(np.abs(R["u"] - 3.0)) < 0.3 and np.nanmax(np.abs(R["v"] + 2.0)) < 0.3


def _gridfit_dense(x, y, z, xl, yl):
    """gridfit.m 'springs' + 'triangle' written out densely, node by node."""
    nx, ny = len(xl), len(yl)
    h = xl[1] - xl[0]
    node = lambda i, j: j + ny * i                       # column-major ny x nx
    rows = []
    for xx, yy, zz in zip(x, y, z):
        i = min(int((xx - xl[0]) // h), nx - 2)
        j = min(int((yy - yl[0]) // h), ny - 2)
        tx, ty = (xx - xl[i]) / h, (yy - yl[j]) / h
        r = np.zeros(nx * ny)
        r[node(i, j)] += 1 - max(tx, ty)
        r[node(i + 1, j + 1)] += min(tx, ty)
        r[node(i + 1, j) if tx > ty else node(i, j + 1)] += abs(tx - ty)
        rows.append(r)
    A = np.array(rows)
    reg = []
    def spring(p, q, s):
        r = np.zeros(nx * ny); r[p] = -s; r[q] = s; reg.append(r)
    for i in range(nx):
        for j in range(ny - 1):
            spring(node(i, j), node(i, j + 1), 1.0)
    for i in range(nx - 1):
        for j in range(ny):
            spring(node(i, j), node(i + 1, j), 1.0)
    d = 1 / np.sqrt(2)
    for i in range(nx - 1):
        for j in range(ny - 1):
            spring(node(i, j), node(i + 1, j + 1), d)
            spring(node(i, j + 1), node(i + 1, j), d)
    R = np.array(reg)
    lam = np.abs(A).sum(0).max() / np.abs(R).sum(0).max()
    sol = np.linalg.lstsq(np.vstack([A, lam * R]), np.r_[z, np.zeros(len(R))], rcond=None)[0]
    return sol.reshape(nx, ny).T


def test_gridfit_scattered_matches_dense_lsq():
    rng = np.random.default_rng(0)
    x = rng.uniform(10.5, 89.5, 300)
    y = rng.uniform(20.5, 69.5, 300)
    z = 2.0 + 0.03 * x - 0.05 * y + 0.1 * np.sin(x / 7.0)
    xl, yl = np.arange(10, 91, 8.0), np.arange(20, 77, 8.0)
    zg = S.gridfit_scattered(x, y, z, xl, yl)
    np.testing.assert_allclose(zg, _gridfit_dense(x, y, z, xl, yl), rtol=0, atol=1e-10)
    # a constant is reproduced exactly; NaN data are dropped
    zc = S.gridfit_scattered(x, y, np.full(300, 3.25), xl, yl)
    np.testing.assert_allclose(zc, 3.25, atol=1e-10)
    zn = z.copy(); zn[::7] = np.nan
    keep = ~np.isnan(zn)
    np.testing.assert_allclose(S.gridfit_scattered(x, y, zn, xl, yl),
                               S.gridfit_scattered(x[keep], y[keep], z[keep], xl, yl), atol=1e-12)
    with pytest.raises(ValueError):
        S.gridfit_scattered(x[:2], y[:2], z[:2], xl, yl)
