"""Oracle (test infrastructure only): restatement of the multigrid integer
search func/funIntegerSearchMg.m, used by tests/ to check the library's
aldic_int_search_mg and the frame's ALDIC_INIT_SEARCH_MG mode.

  * level 1 (funIntegerSearchMg.m:19-35): the ROI trimmed by
    borderGap = 1 + round(0.75 w); normxcorr2 of the whole f ROI against the
    same g ROI; findpeak over the full map gives one global shift
  * shift the g ROI by ceil(shift), clamp it to the border and shrink f to
    match; make both widths even (:37-54)
  * levels 2.. (:56-200): split every region in x, in y or in both (by the
    nominal width ratio; a region is split only while its own width exceeds
    w), correlate f(region) against g(region +- 5 px), findpeak on the
    13 x 14 crop of the map, accumulate the offsets; a region whose
    correlation raises (out of the image, constant template, NaN bounds)
    becomes NaN (Phi 0); between levels the g regions follow ceil(u), are
    clamped and made even as on level 1
  * last level: compute_qFactor on each full map, normalised over regions
  * node grid (:216-244): borders from the displacements of the extreme
    regions, xList = gridx(1):step:gridx(2), and gridfit 'springs' (triangle
    interpolation, smoothness 1; func/gridfit.m:295-298,484-493,523-596) of
    u, v, Phi and the q-factors at the region centres strictly inside the
    grid; NaN data are dropped per field (gridfit.m:332-337).

normxcorr2, findpeak and compute_qFactor are the C oracle's (the same
restatements the uniform search uses).  scipy's sparse direct solve of the
regularised normal equations stands in for gridfit's backslash.
"""
from __future__ import annotations

import math

import numpy as np

from . import _DT, _c, _p, lib


def _round(x):
    """MATLAB round: half away from zero."""
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def _ceil(x):
    return math.ceil(x) if np.isfinite(x) else float("nan")


def _ncc(f, g, dt, mu_g, trect, drect, ox, oy):
    """normxcorr2 restated over the offsets ox[0]..ox[1] x oy[0]..oy[1];
    None when normxcorr2 would raise."""
    import ctypes as C
    H, W = f.shape
    nr, nc = ox[1] - ox[0] + 1, oy[1] - oy[0] + 1
    out = np.empty(nr * nc)
    tr = np.asarray(trect, np.int32)
    dr = np.asarray(drect, np.int32)
    rc = lib().orc_ncc_map(_p(f), _p(g), dt, W, H, C.c_double(mu_g), _p(tr), _p(dr),
                           ox[0], ox[1], oy[0], oy[1], _p(out))
    if rc:
        return None
    return out


def findpeak(m, nr, nc):
    out = np.empty(3)
    lib().orc_findpeak(_p(np.ascontiguousarray(m)), nr, nc, _p(out))
    return out


def qfactor(m):
    out = np.empty(2)
    lib().orc_qfactor(_p(np.ascontiguousarray(m)), len(m), _p(out))
    return out


def _valid_rect(r, W, H):
    x1, x2, y1, y2 = r
    if not all(np.isfinite(v) for v in r):
        return False
    if x1 != int(x1) or x2 != int(x2) or y1 != int(y1) or y2 != int(y2):
        return False
    return 1 <= x1 <= x2 <= W and 1 <= y1 <= y2 <= H


def _clamp_even(xf, yf, xg, yg, bg, W, H):
    """funIntegerSearchMg.m:37-54 / :180-208 on one region (in place)."""
    if xg[0] < bg:
        t = xg[0]; xg[0] = bg; xf[0] = xf[0] + bg - t
    if yg[0] < bg:
        t = yg[0]; yg[0] = bg; yf[0] = yf[0] + bg - t
    if xg[1] > W - bg:
        t = xg[1]; xg[1] = W - bg; xf[1] = xf[1] + (W - bg) - t
    if yg[1] > H - bg:
        t = yg[1]; yg[1] = H - bg; yf[1] = yf[1] + (H - bg) - t


def _make_even(xf, yf, xg, yg):
    d = xf[1] - xf[0]
    if np.isfinite(d) and d % 2 == 1:
        xf[1] -= 1; xg[1] -= 1
    d = yf[1] - yf[0]
    if np.isfinite(d) and d % 2 == 1:
        yf[1] -= 1; yg[1] -= 1


def regions(f, g, gridx, gridy, winsize, mu_g):
    """Levels of funIntegerSearchMg.m:9-209.  Returns the last level's regions
    (f ranges, 1-based inclusive), u, v, Phi, normalised q-factors and the
    trimmed gridx, gridy."""
    H, W = f.shape
    f = _c(f)
    g = _c(g)
    dt = _DT[f.dtype]
    w = winsize
    bg = 1 + _round(0.75 * w)
    gx, gy = list(gridx), list(gridy)
    if gx[0] < bg: gx[0] = bg
    if gy[0] < bg: gy[0] = bg
    if gx[1] > W - bg: gx[1] = W - bg
    if gy[1] > H - bg: gy[1] = H - bg
    a, b = gx[1] - gx[0] + 1, gy[1] - gy[0] + 1
    rect = [gx[0], gx[1], gy[0], gy[1]]
    m = _ncc(f, g, dt, mu_g, rect, rect, (-(a - 1), a - 1), (-(b - 1), b - 1))
    if m is None:
        raise ValueError("normxcorr2: the ROI template is constant")
    r, c, _ = findpeak(m, 2 * a - 1, 2 * b - 1)
    ut, vt = r - a, c - b
    level1 = (ut, vt)
    xf, yf = [float(gx[0]), float(gx[1])], [float(gy[0]), float(gy[1])]
    xg = [gx[0] + _ceil(ut), gx[1] + _ceil(ut)]
    yg = [gy[0] + _ceil(vt), gy[1] + _ceil(vt)]
    _clamp_even(xf, yf, xg, yg, bg, W, H)
    _make_even(xf, yf, xg, yg)
    R = [(xf, yf, xg, yg)]
    ucur, vcur = [_ceil(ut)], [_ceil(vt)]
    wx, wy = xf[1] - xf[0], yf[1] - yf[0]
    ratio = wx / wy
    while True:
        new, un, vn = [], [], []
        if ratio > 2:
            wx = wx / 2
            for (xf, yf, xg, yg), u0, v0 in zip(R, ucur, vcur):
                if xf[1] - xf[0] > w:
                    mf, mg = 0.5 * (xf[0] + xf[1]), 0.5 * (xg[0] + xg[1])
                    new += [([xf[0], mf], yf[:], [xg[0], mg], yg[:]),
                            ([mf, xf[1]], yf[:], [mg, xg[1]], yg[:])]
                else:
                    new += [(xf[:], yf[:], xg[:], yg[:])] * 2
                un += [u0] * 2; vn += [v0] * 2
        elif ratio < 0.5:
            wy = wy / 2
            for (xf, yf, xg, yg), u0, v0 in zip(R, ucur, vcur):
                if yf[1] - yf[0] > w:
                    mf, mg = 0.5 * (yf[0] + yf[1]), 0.5 * (yg[0] + yg[1])
                    new += [(xf[:], [yf[0], mf], xg[:], [yg[0], mg]),
                            (xf[:], [mf, yf[1]], xg[:], [mg, yg[1]])]
                else:
                    new += [(xf[:], yf[:], xg[:], yg[:])] * 2
                un += [u0] * 2; vn += [v0] * 2
        else:
            wx, wy = wx / 2, wy / 2
            for (xf, yf, xg, yg), u0, v0 in zip(R, ucur, vcur):
                if xf[1] - xf[0] > w and yf[1] - yf[0] > w:
                    mxf, mxg = 0.5 * (xf[0] + xf[1]), 0.5 * (xg[0] + xg[1])
                    myf, myg = 0.5 * (yf[0] + yf[1]), 0.5 * (yg[0] + yg[1])
                    xs_f, xs_g = [[xf[0], mxf], [mxf, xf[1]]], [[xg[0], mxg], [mxg, xg[1]]]
                    ys_f, ys_g = [[yf[0], myf], [myf, yf[1]]], [[yg[0], myg], [myg, yg[1]]]
                    for jy in range(2):
                        for ix in range(2):
                            new.append((xs_f[ix][:], ys_f[jy][:], xs_g[ix][:], ys_g[jy][:]))
                else:
                    new += [(xf[:], yf[:], xg[:], yg[:])] * 4
                un += [u0] * 4; vn += [v0] * 4
        last = wx < w and wy < w
        n = len(new)
        u = np.array(un, float)
        v = np.array(vn, float)
        phi = np.zeros(n)
        qf = np.full((n, 2), np.nan)
        for t, (xf, yf, xg, yg) in enumerate(new):
            trect = [xf[0], xf[1], yf[0], yf[1]]
            drect = [xg[0] - 5, xg[1] + 5, yg[0] - 5, yg[1] + 5]
            ok = _valid_rect(trect, W, H) and _valid_rect(drect, W, H)
            if ok:
                trect = [int(q) for q in trect]
                drect = [int(q) for q in drect]
                a, b = trect[1] - trect[0] + 1, trect[3] - trect[2] + 1
                ok = a * b >= 2
            if ok:
                if last:
                    dw, dh = drect[1] - drect[0] + 1, drect[3] - drect[2] + 1
                    full = _ncc(f, g, dt, mu_g, trect, drect, (-(a - 1), dw - 1), (-(b - 1), dh - 1))
                    ok = full is not None
                    if ok:
                        qf[t] = qfactor(full)
                        fr = a + dw - 1
                        crop = full.reshape(b + dh - 1, fr)[b - 2:b + 12, a - 2:a + 11]
                        crop = np.ascontiguousarray(crop).reshape(-1)
                else:
                    crop = _ncc(f, g, dt, mu_g, trect, drect, (-1, 11), (-1, 12))
                    ok = crop is not None
            if ok:
                r, c, mx = findpeak(crop, 13, 14)
                u[t] += r - 7
                v[t] += c - 7
                phi[t] = mx
            else:
                u[t] = v[t] = np.nan
                phi[t] = 0.0
                qf[t] = np.nan
        if last:
            for k in range(2):
                q = qf[:, k] - np.nanmin(qf[:, k])
                qf[:, k] = q / np.nanmax(q)
            return dict(regions=new, u=u, v=v, phi=phi, qf=qf, gridx=gx, gridy=gy,
                        level1=level1, failed=int(np.isnan(u).sum()))
        R = []
        for (xf, yf, _, _), uk, vk in zip(new, u, v):
            xg = [xf[0] + _ceil(uk), xf[1] + _ceil(uk)]
            yg = [yf[0] + _ceil(vk), yf[1] + _ceil(vk)]
            xf, yf = xf[:], yf[:]
            _clamp_even(xf, yf, xg, yg, bg, W, H)
            R.append((xf, yf, xg, yg))
        for xf, yf, xg, yg in R:
            _make_even(xf, yf, xg, yg)
        ratio = wx / wy
        ucur = [_ceil(q) for q in u]
        vcur = [_ceil(q) for q in v]


def springs_norm1(nx, ny):
    """norm(Areg, 1) of the springs regularizer on a uniform grid."""
    d = 1.0 / math.sqrt(2.0)
    if nx >= 3 and ny >= 3:
        return 4 + 4 * d
    best = 0.0
    for i in range(nx):
        for j in range(ny):
            s = (i > 0) + (i < nx - 1) + (j > 0) + (j < ny - 1)
            s += d * ((i > 0 and j > 0) + (i < nx - 1 and j > 0) + (i > 0 and j < ny - 1)
                      + (i < nx - 1 and j < ny - 1))
            best = max(best, s)
    return best


def gridfit_scattered(x, y, z, xnodes, ynodes):
    """gridfit(x, y, z, xnodes, ynodes, 'regularizer', 'springs') with the
    defaults smoothness 1, interp 'triangle', autoscale 'on' on uniform
    nodes (gridfit.m:328-596).  Returns the ny x nx grid (rows = y)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    x, y, z = (np.asarray(q, float).reshape(-1) for q in (x, y, z))
    k = np.isnan(x) | np.isnan(y) | np.isnan(z)
    x, y, z = x[~k], y[~k], z[~k]
    n = len(x)
    if n < 3:
        raise ValueError("gridfit: insufficient data")
    xn, yn = np.asarray(xnodes, float), np.asarray(ynodes, float)
    nx, ny = len(xn), len(yn)
    if x.min() < xn[0] or x.max() > xn[-1] or y.min() < yn[0] or y.max() > yn[-1]:
        raise ValueError("gridfit: data outside the nodes")
    dx, dy = np.diff(xn), np.diff(yn)
    # histc: last node -> last cell
    ix = np.clip(np.searchsorted(xn, x, side="right") - 1, 0, nx - 2)
    iy = np.clip(np.searchsorted(yn, y, side="right") - 1, 0, ny - 2)
    tx = np.clip((x - xn[ix]) / dx[ix], 0, 1)
    ty = np.clip((y - yn[iy]) / dy[iy], 0, 1)
    ind = iy + ny * ix                                   # 0-based, column-major ny x nx
    L = np.where(tx > ty, ny, 1)
    t1, t2 = np.minimum(tx, ty), np.maximum(tx, ty)
    rows = np.repeat(np.arange(n), 3)
    cols = np.stack([ind, ind + ny + 1, ind + L], 1).reshape(-1)
    vals = np.stack([1 - t2, t1, t2 - t1], 1).reshape(-1)
    ng = nx * ny
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, ng))
    # springs (unit axial stiffness, 1/sqrt(2) diagonals on a uniform grid)
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    gi = lambda i, j: j + ny * i
    pairs, st = [], []
    m = J < ny - 1
    pairs.append((gi(I[m], J[m]), gi(I[m], J[m] + 1))); st.append(1.0)
    m = I < nx - 1
    pairs.append((gi(I[m], J[m]), gi(I[m] + 1, J[m]))); st.append(1.0)
    m = (I < nx - 1) & (J < ny - 1)
    pairs.append((gi(I[m], J[m]), gi(I[m] + 1, J[m] + 1))); st.append(1 / math.sqrt(2))
    pairs.append((gi(I[m], J[m] + 1), gi(I[m] + 1, J[m]))); st.append(1 / math.sqrt(2))
    rr, cc, vv, r0 = [], [], [], 0
    for (p, q), s in zip(pairs, st):
        k = len(p)
        rr += [np.arange(r0, r0 + k)] * 2
        cc += [p, q]
        vv += [np.full(k, -s), np.full(k, s)]
        r0 += k
    Areg = sp.csr_matrix((np.concatenate(vv), (np.concatenate(rr), np.concatenate(cc))),
                         shape=(r0, ng))
    NA = abs(A).sum(0).max()
    NR = springs_norm1(nx, ny)
    lam = NA / NR
    N = (A.T @ A + (lam * lam) * (Areg.T @ Areg)).tocsc()
    zg = spl.spsolve(N, A.T @ z)
    return zg.reshape(nx, ny).T


def int_search_mg(f, g, gridx, gridy, winsize, step, mu_g=None):
    """[x, y, u, v, cc] = funIntegerSearchMg(f, g, gridx, gridy, winsize,
    step, step) on raw images (D padded with mu_g, zero in normalised
    units).  Arrays are ny x nx (rows = y)."""
    from . import normalize
    if mu_g is None:
        _, mu_g, _ = normalize(g)
    H, W = f.shape
    R = regions(f, g, gridx, gridy, winsize, mu_g)
    reg = R["regions"]
    tx = np.array([0.5 * (q[0][0] + q[0][1]) for q in reg])
    ty = np.array([0.5 * (q[1][0] + q[1][1]) for q in reg])
    u, v, phi, qf = R["u"], R["v"], R["phi"], R["qf"]
    gx, gy = list(R["gridx"]), list(R["gridy"])
    ix1, ix2 = int(np.argmin(tx)), int(np.argmax(tx))
    iy1, iy2 = int(np.argmin(ty)), int(np.argmax(ty))
    bx1 = math.ceil(1 + 1.25 * winsize + u[ix1]) if np.isfinite(u[ix1]) else np.nan
    bx2 = math.ceil(1 + 1.25 * winsize + u[ix2]) if np.isfinite(u[ix2]) else np.nan
    by1 = math.ceil(1 + 1.25 * winsize + v[iy1]) if np.isfinite(v[iy1]) else np.nan
    by2 = math.ceil(1 + 1.25 * winsize + v[iy2]) if np.isfinite(v[iy2]) else np.nan
    if gx[0] < bx1: gx[0] = bx1
    if gy[0] < by1: gy[0] = by1
    if gx[1] > W - bx2 + 1: gx[1] = W - bx2 + 1
    if gy[1] > H - by2 + 1: gy[1] = H - by2 + 1
    xl = np.arange(gx[0], gx[1] + 1, step, dtype=float)
    yl = np.arange(gy[0], gy[1] + 1, step, dtype=float)
    sel = (tx > xl.min()) & (tx < xl.max()) & (ty > yl.min()) & (ty < yl.max())
    fit = lambda z: gridfit_scattered(tx[sel], ty[sel], z[sel], xl, yl)
    X, Y = np.meshgrid(xl, yl)
    return dict(x=X, y=Y, u=fit(u), v=fit(v), ccmax=fit(phi), q1=fit(qf[:, 0]), q2=fit(qf[:, 1]),
                xlist=xl, ylist=yl, regions=R)
