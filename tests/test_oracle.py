"""The CPU oracle, pinned against the reference's own code (ba_interp2) and
against known-answer tests written from each algorithm's definition (the
MATLAB parts of the reference cannot run here)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))


# ------------------------------------------------------------------ a3
def test_interp_matches_reference_golden(oracle):
    g = np.load(os.path.join(HERE, "golden", "ba_interp2_ref.npz"))
    for t in ("f64", "f32"):
        z = oracle.ba_interp2(g[f"F_{t}"], g[f"X_{t}"], g[f"Y_{t}"])
        assert z.dtype == g[f"Z_{t}"].dtype
        np.testing.assert_array_equal(z, g[f"Z_{t}"])
        z1 = oracle.ba_interp2(g[f"F_{t}"][0], g[f"X_{t}"], g[f"Y_{t}"])
        np.testing.assert_array_equal(z1, g[f"Z1_{t}"])


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference not compiled")
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_interp_matches_reference_live(oracle, dt):
    rng = np.random.default_rng(1)
    F = rng.uniform(0, 255, (64, 48)).astype(dt)
    X = rng.uniform(-5, 70, 5000).astype(dt)
    Y = rng.uniform(-5, 55, 5000).astype(dt)
    np.testing.assert_array_equal(oracle.ba_interp2(F, X, Y), oracle.ref_ba_interp2(F, X, Y))


def test_interp_nonfinite_gives_nan(oracle):
    F = np.arange(20.0).reshape(4, 5)
    z = oracle.ba_interp2(F, np.array([np.nan, 2.0, np.inf]), np.array([2.0, np.nan, 1.0]))
    assert np.isnan(z).all()


# ------------------------------------------------------------------ a1/a2
def test_normalize_kat(oracle):
    rng = np.random.default_rng(2)
    img = rng.integers(0, 256, (40, 50), dtype=np.uint8)
    out, m, s = oracle.normalize(img, [3, 45, 5, 30])
    roi = img[4:30, 2:45].astype(float)
    assert m == pytest.approx(roi.mean(), rel=1e-14)
    assert s == pytest.approx(roi.std(ddof=1), rel=1e-13)
    np.testing.assert_allclose(out, (img - roi.mean()) / roi.std(ddof=1), rtol=1e-12, atol=1e-13)


def test_gradient_kat(oracle):
    rng = np.random.default_rng(3)
    f = rng.standard_normal((30, 40))
    f[10:20, 10:25] = 0.75  # flat patch: exact zeros required by funICGN.m:54
    mask = np.ones_like(f)
    mask[25:, :] = 0
    dx, dy = oracle.gradient(f, mask)
    h = np.array([-1 / 60, 3 / 20, -3 / 4, 0, 3 / 4, -3 / 20, 1 / 60])
    ex = np.zeros_like(f)
    ey = np.zeros_like(f)
    for k, c in enumerate(h):
        o = k - 3
        ex[3:-3, 3:-3] += c * f[3:-3, 3 + o:f.shape[1] - 3 + o]
        ey[3:-3, 3:-3] += c * f[3 + o:f.shape[0] - 3 + o, 3:-3]
    ex *= mask
    ey *= mask
    np.testing.assert_allclose(dx, ex, atol=1e-14)
    np.testing.assert_allclose(dy, ey, atol=1e-14)
    assert (dx[13:17, 13:22] == 0).all() and (dy[13:17, 13:22] == 0).all()
    assert (dx[25:] == 0).all()


# ------------------------------------------------------------------ a4/a5
def _normxcorr2_def(T, D, pad):
    """Normalised cross-correlation from its definition: template T over D
    padded with `pad` outside; full map of shape (T+D-1)."""
    th, tw = T.shape
    dh, dw = D.shape
    P = np.full((dh + 2 * th - 2, dw + 2 * tw - 2), float(pad))
    P[th - 1:th - 1 + dh, tw - 1:tw - 1 + dw] = D
    Tz = T - T.mean()
    out = np.zeros((dh + th - 1, dw + tw - 1))
    for a in range(out.shape[0]):
        for b in range(out.shape[1]):
            A = P[a:a + th, b:b + tw]
            Az = A - A.mean()
            den = np.sqrt((Tz * Tz).sum() * (Az * Az).sum())
            out[a, b] = (Tz * Az).sum() / den if den > 0 else 0.0
    return out


def _findpeak_lstsq(f):
    imax = np.argmax(f.ravel(order="F"))
    r, c = imax % f.shape[0], imax // f.shape[0]
    if r in (0, f.shape[0] - 1) or c in (0, f.shape[1] - 1):
        return r + 1.0, c + 1.0, f[r, c]
    u = f[r - 1:r + 2, c - 1:c + 2].ravel(order="F")
    x = np.array([-1, -1, -1, 0, 0, 0, 1, 1, 1.0])
    y = np.array([-1, 0, 1, -1, 0, 1, -1, 0, 1.0])
    X = np.stack([np.ones(9), x, y, x * y, x * x, y * y], 1)
    A = np.linalg.lstsq(X, u, rcond=None)[0]
    xo = (-A[2] * A[3] + 2 * A[5] * A[1]) / (A[3] ** 2 - 4 * A[4] * A[5])
    yo = -1 / (A[3] ** 2 - 4 * A[4] * A[5]) * (A[3] * A[1] - 2 * A[4] * A[2])
    if abs(xo) > 1 or abs(yo) > 1:
        return r + 1.0, c + 1.0, f[r, c]
    return (r + 1) + yo, (c + 1) + xo, (xo, yo)


def test_int_search_kat(oracle, synth):
    W = H = 96
    f = synth.speckle(W, H, 300, 11)
    g = synth.warp(f, synth.uniform_affine(0.0, 0.0, 2.3, -1.6), 1.0, 11)
    w, step, s = 12, 8, 5
    x, y, u, v, cc, q = oracle.int_search(f, g, g.astype(float).mean(), [1, W], [1, H], w, step,
                                          [s, s], qfactors=True)
    ny, nx = u.shape
    _, _, x1, y1 = oracle.search_dims(W, H, [1, W], [1, H], w, step, [s, s])
    mu = g.astype(float).mean()
    checked = 0
    for iy in range(ny):
        for ix in range(nx):
            ii, jj = x1 + ix * step, y1 + iy * step
            T = f[jj - 1:jj + w, ii - 1:ii + w].T.astype(float)     # MATLAB (x, y) order
            D = g[jj - 1 - s:jj + w + s, ii - 1 - s:ii + w + s].T.astype(float)
            full = _normxcorr2_def(T, D, mu)
            crop = full[w - 1:full.shape[0] - w + 1, w - 1:full.shape[1] - w + 1]
            r, c, _ = _findpeak_lstsq(crop)
            assert x[iy, ix] == (ii + ii + w) / 2 and y[iy, ix] == (jj + jj + w) / 2
            assert abs(u[iy, ix] - (r - (s + 2))) < 1.5e-3
            assert abs(v[iy, ix] - (c - (s + 2))) < 1.5e-3
            checked += 1
    assert checked == nx * ny > 10
    # the applied shift is recovered to within the interpolation/noise error
    assert np.nanmedian(np.abs(u - 2.3)) < 0.15 and np.nanmedian(np.abs(v + 1.6)) < 0.15
    assert q.shape == (nx * ny, 2) and np.nanmax(q) == pytest.approx(1.0)


def test_search_dims_trimming(oracle):
    # plain 512^2 workload: gridx trimmed to [31, 462], XList = 31:10:451
    nx, ny, x1, y1 = oracle.search_dims(512, 512, [1, 512], [1, 512], 20, 10, [20, 20])
    assert (nx, ny, x1, y1) == (43, 43, 31, 31)


def test_flat_template_gives_nan(oracle):
    f = np.full((64, 64), 7, np.uint8)
    g = np.random.default_rng(0).integers(0, 255, (64, 64)).astype(np.uint8)
    x, y, u, v, cc, q = oracle.int_search(f, g, 100.0, [1, 64], [1, 64], 10, 10, [4, 4], True)
    assert np.isnan(u).all() and np.isnan(cc).all() and np.isnan(q).all()


# ------------------------------------------------------------------ a7-a9
def _prepared(oracle, synth, W=160, H=140, shift=(0.37, -0.61), seed=5):
    f = synth.speckle(W, H, 900, seed)
    g = synth.warp(f, synth.uniform_affine(0.0, 0.0, *shift), 0.5, seed)
    fn, _, _ = oracle.normalize(f)
    gn, _, _ = oracle.normalize(g)
    dx, dy = oracle.gradient(fn)
    return fn, gn, dx, dy


def test_icgn_recovers_translation(oracle, synth):
    fn, gn, dx, dy = _prepared(oracle, synth)
    xs = np.arange(40, 121, 20.0)
    X, Y = np.meshgrid(xs, xs[:4])
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    U0 = np.zeros(2 * len(coords))
    U, F, it, H21 = oracle.icgn_batch(fn, gn, dx, dy, coords, U0, 20, 1e-3)
    assert ((it >= 1) & (it <= 100)).all()
    np.testing.assert_allclose(U[0::2], 0.37, atol=0.02)
    np.testing.assert_allclose(U[1::2], -0.61, atol=0.02)
    assert np.abs(F).max() < 5e-3
    # H21 is the lower triangle of a symmetric positive definite 6x6
    for j in range(len(coords)):
        Hm = np.zeros((6, 6))
        k = 0
        for c in range(6):
            for r in range(c, 6):
                Hm[r, c] = Hm[c, r] = H21[k, j]
                k += 1
        assert np.linalg.eigvalsh(Hm).min() > 0


def test_icgn_status_codes(oracle, synth):
    fn, gn, dx, dy = _prepared(oracle, synth)
    dx2 = dx.copy()
    dx2[60:100, 60:100] = 0.0  # masked area -> 102
    coords = np.array([[5.0, 50.0], [80.0, 80.0], [40.5, 50.0], [40.0, 60.0]])
    U0 = np.zeros(8)
    U, F, it, H21 = oracle.icgn_batch(fn, gn, dx2, dy, coords, U0, 20, 1e-3)
    assert it[0] == -1 and np.isnan(U[0]) and np.isnan(F[0]) and (H21[:, 0] == 0).all()
    assert it[1] == 102 and U[2] == 0 and (H21[:, 1] == 0).all()
    assert it[2] == -1                       # half-integer subset bounds
    assert 1 <= it[3] <= 100
    # a guess that walks the subset out of the image -> 101
    U0b = np.array([0.0, 0.0, 0.0, 0.0, -200.0, 0.0, 0.0, 0.0])
    _, _, it2, _ = oracle.icgn_batch(fn, gn, dx, dy, coords, U0b, 20, 1e-3)
    assert it2[2] == -1 and it2[0] == -1


def test_subpb1_pulls_to_penalty(oracle, synth):
    fn, gn, dx, dy = _prepared(oracle, synth)
    coords = np.array([[60.0, 60.0], [100.0, 80.0]])
    U0 = np.zeros(4)
    U, F, it, H21 = oracle.icgn_batch(fn, gn, dx, dy, coords, U0, 20, 1e-4)
    Ub, itb = oracle.subpb1_batch(fn, gn, dx, dy, coords, U, F, np.zeros(4), H21, 20, 1e-3, 1e-4)
    np.testing.assert_allclose(Ub, U, atol=5e-3)
    # The penalty mu*(P - UOld - vdual) enters b like the image term and the
    # step is applied inverse-compositionally (funICGN_Subpb1.m:269,285,311-329),
    # so it moves P AWAY from UOld + vdual, by about mu/H2 * vdual.  This is the
    # reference's behaviour and the restatement keeps it.
    vd = np.array([0.2, 0.1, -0.1, 0.3])
    Ua, _ = oracle.subpb1_batch(fn, gn, dx, dy, coords, U, F, np.zeros(4), H21, 20, 1e-2, 1e-6)
    Uc, _ = oracle.subpb1_batch(fn, gn, dx, dy, coords, U, F, vd, H21, 20, 1e-2, 1e-6)
    d = Uc - Ua
    assert (d * vd < 0).all() and np.abs(d).max() < 0.1 * np.abs(vd).max()


# ------------------------------------------------------------------ a10/a11
def _subpb2_scipy(M, N, h, beta, mu, U, F, ud, vd):
    """Independent restatement of Subpb2.m:76-195 with scipy sparse."""
    A, b = subpb2_system(M, N, h, beta, mu, U, F, ud, vd)
    return spla.spsolve(A.tocsc(), b)


def subpb2_system(M, N, h, beta, mu, U, F, ud, vd):
    """The sparse matrix (2n x 2n, DOFs [u1 v1 u2 v2 ...]) and right-hand side
    Subpb2.m:76-163 assembles on the uniform M x N mesh."""
    n = M * N
    gp = [-np.sqrt(3 / 5), 0, np.sqrt(3 / 5)]
    gw = [5 / 9, 8 / 9, 5 / 9]
    rows, cols, vals = [], [], []
    b = np.zeros(2 * n)
    for ej in range(N - 1):
        for ei in range(M - 1):
            nd = [ej * M + ei, ej * M + ei + 1, (ej + 1) * M + ei + 1, (ej + 1) * M + ei]
            px = np.array([(q % M) * h for q in nd])
            py = np.array([(q // M) * h for q in nd])
            idx = np.array([[2 * q, 2 * q + 1] for q in nd]).ravel()
            FW = np.array([[F[4 * q + 0] - ud[4 * q + 0], F[4 * q + 2] - ud[4 * q + 2],
                            F[4 * q + 1] - ud[4 * q + 1], F[4 * q + 3] - ud[4 * q + 3]]
                           for q in nd for _ in (0, 1)])
            UV = U[idx] - vd[idx]
            A8 = np.zeros((8, 8))
            b8 = np.zeros(8)
            for ti in range(3):
                for tj in range(3):
                    k, e = gp[ti], gp[tj]
                    Nn = np.array([(1 - k) * (1 - e), (1 + k) * (1 - e), (1 + k) * (1 + e),
                                   (1 - k) * (1 + e)]) / 4
                    dk = np.array([-(1 - e), 1 - e, 1 + e, -(1 + e)]) / 4
                    de = np.array([-(1 - k), -(1 + k), 1 + k, 1 - k]) / 4
                    J = np.array([[dk @ px, dk @ py], [de @ px, de @ py]])
                    Ji = np.linalg.inv(J)
                    g = Ji @ np.stack([dk, de])
                    DN = np.zeros((4, 8))
                    DN[0, 0::2] = g[0]; DN[1, 0::2] = g[1]
                    DN[2, 1::2] = g[0]; DN[3, 1::2] = g[1]
                    Nm = np.zeros((2, 8))
                    Nm[0, 0::2] = Nn; Nm[1, 1::2] = Nn
                    s = np.linalg.det(J) * gw[ti] * gw[tj]
                    A8 += s * (beta * DN.T @ DN + mu * Nm.T @ Nm)
                    b8 += s * (beta * np.diag(DN.T @ FW.T) + mu * Nm.T @ Nm @ UV)
            for r in range(8):
                b[idx[r]] += b8[r]
                for q in range(8):
                    rows.append(idx[r]); cols.append(idx[q]); vals.append(A8[r, q])
    A = sp.csr_matrix((vals, (rows, cols)), shape=(2 * n, 2 * n))
    return A, b


def test_subpb2_matches_sparse_restatement(oracle):
    rng = np.random.default_rng(7)
    M, N, h = 9, 7, 8.0
    n = M * N
    U = rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    ud = 0.001 * rng.standard_normal(4 * n)
    vd = 0.01 * rng.standard_normal(2 * n)
    for beta in (1e-3 * h * h * 1e-3, 0.1 * h * h * 1e-3):
        x, it = oracle.subpb2(M, N, h, beta, 1e-3, U, F, ud, vd)
        ref = _subpb2_scipy(M, N, h, beta, 1e-3, U, F, ud, vd)
        np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-11)


def test_nodal_strain_linear_field(oracle):
    M, N, h = 6, 5, 10.0
    xs = np.arange(M) * h
    ys = np.arange(N) * h
    X, Y = np.meshgrid(xs, ys)
    X, Y = X.ravel(), Y.ravel()
    U = np.empty(2 * M * N)
    U[0::2] = 0.01 * X + 0.002 * Y
    U[1::2] = -0.003 * X + 0.005 * Y
    F = oracle.nodal_strain(M, N, h, U)
    # slots as funGlobal_NodalStrainAvg.m writes them: du/dx du/dy dv/dx dv/dy
    np.testing.assert_allclose(F[0::4], 0.01, atol=1e-14)
    np.testing.assert_allclose(F[1::4], 0.002, atol=1e-14)
    np.testing.assert_allclose(F[2::4], -0.003, atol=1e-14)
    np.testing.assert_allclose(F[3::4], 0.005, atol=1e-14)


# ------------------------------------------------------------------ grid solvers
def _springs_ls(M, N, d):
    """gridfit.m 'springs' least squares written out with scipy (smoothness 1)."""
    n = M * N
    ok = ~np.isnan(d)
    A = sp.csr_matrix((np.ones(ok.sum()), (np.arange(ok.sum()), np.nonzero(ok)[0])),
                      shape=(ok.sum(), n))
    rows = []

    def spring(a, b, k):
        rows.append((a, b, k))

    for j in range(N):
        for i in range(M):
            k = j * M + i
            if i < M - 1:
                spring(k, k + 1, 1.0)
            if j < N - 1:
                spring(k, k + M, 1.0)
            if i < M - 1 and j < N - 1:
                spring(k, k + M + 1, 1 / np.sqrt(2))
                spring(k + 1, k + M, 1 / np.sqrt(2))
    r = np.arange(len(rows))
    a = np.array([t[0] for t in rows]); b = np.array([t[1] for t in rows])
    kk = np.array([t[2] for t in rows])
    R = sp.csr_matrix((np.r_[-kk, kk], (np.r_[r, r], np.r_[a, b])), shape=(len(rows), n))
    NA = abs(A).sum(0).max()
    NR = abs(R).sum(0).max()
    big = sp.vstack([A, R * (NA / NR)])
    rhs = np.r_[d[ok], np.zeros(len(rows))]
    return spla.lsqr(big, rhs, atol=1e-15, btol=1e-15, iter_lim=100000)[0]


def test_gridfit_springs_matches_lsq(oracle):
    rng = np.random.default_rng(8)
    M, N = 11, 8
    d = np.sin(np.arange(M * N) * 0.3) + 0.1 * rng.standard_normal(M * N)
    d[[3, 17, 40, 41, 42]] = np.nan
    z = oracle.gridfit_springs(M, N, d[None])[0]
    np.testing.assert_allclose(z, _springs_ls(M, N, d), atol=1e-8)


def test_inpaint_springs_harmonic(oracle):
    M, N = 9, 7
    X, Y = np.meshgrid(np.arange(M), np.arange(N))
    z = (2.0 * X - 0.5 * Y + 3).ravel().astype(float)  # harmonic: kept exactly
    zn = z.copy()
    zn[[10, 11, 20, 30, 31, 32]] = np.nan
    out = oracle.inpaint_springs(M, N, zn)
    np.testing.assert_allclose(out, z, atol=1e-10)


def test_localicgn_post_flags(oracle):
    M, N = 5, 4
    it = np.array([3] * 20, np.int32)
    it[[2, 7]] = [101, 9]
    U = np.arange(40, dtype=float)
    F = np.zeros(80)
    U2, F2, nb = oracle.localicgn_post(M, N, it, U, F)
    assert nb == 1  # the 101 only; the 9 is removed by the 0.15-sigma flag
    assert not np.isnan(U2).any()
    keep = np.setdiff1d(np.arange(20), [2, 7])
    np.testing.assert_array_equal(U2[2 * keep], U[2 * keep])


# ------------------------------------------------------------------ a12
def test_frame_plain512_accuracy(oracle, synth):
    wl = synth.workload("plain512")
    f, g = wl.images()
    r = oracle.frame(f, g, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3)
    ut, vt = synth.truth(wl, r["x0"], r["y0"])
    e = np.r_[r["U"][0::2] - ut, r["U"][1::2] - vt]
    assert np.sqrt(np.mean(e ** 2)) < 0.01
    assert r["admm_steps"] == 3 and r["beta"] > 0
    np.testing.assert_allclose(np.mean(r["F"][0::4]), 0.01, atol=5e-4)
    np.testing.assert_allclose(np.mean(r["F"][3::4]), 0.005, atol=5e-4)
