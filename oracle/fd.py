"""Oracle (test infrastructure only): numpy/scipy restatement of the
finite-difference variant of Subproblem 2, used by tests/ to check the
library's FD path.

  * derivative_op  func/funDerivativeOp.m:1-47: the sparse 4MN x 2MN operator
    (rows F11 F21 F12 F22 per node, central differences / 2h, one-sided and
    doubled where a neighbour is missing; duplicate entries summed as
    MATLAB's sparse() does)
  * subpb2_fd      main_ALDIC.m:243-259 / :386-390: (beta D'D + mu I) on the
    interior (M-2) x (N-2) nodes (funFDNeumannBCInd.m), border nodes keep U;
    scipy's sparse direct solve stands in for MATLAB's backslash
  * frame_fd       one frame of main_ALDIC.m with DICpara.Subpb2FDOrFEM = 1,
    built from the C oracle's search / IC-GN / Subpb1 pieces, with the
    reference's ROI and (optionally) its in-loop smoothing
"""
from __future__ import annotations

import numpy as np


def derivative_op(M, N, h):
    import scipy.sparse as sp
    k = np.arange(M * N)
    x, y = k % M, k // M                                 # x fastest (ndgrid(1:M,1:N))
    idx = k + 1                                          # 1-based node index
    back = np.where(y == N - 1, idx, idx + M)
    front = np.where(y == 0, idx, idx - M)
    right = np.where(x == M - 1, idx, idx + 1)
    left = np.where(x == 0, idx, idx - 1)
    rows = (4 * idx[:, None] + np.arange(-3, 1)[None, :])            # F11 F21 F12 F22
    col1 = np.stack([2 * left - 1, 2 * left, 2 * front - 1, 2 * front], 1)
    col2 = np.stack([2 * right - 1, 2 * right, 2 * back - 1, 2 * back], 1)
    v1 = -np.ones((M * N, 4))
    v2 = np.ones((M * N, 4))
    bx = (x == 0) | (x == M - 1)
    by = (y == 0) | (y == N - 1)
    v1[bx, 0:2] = -2
    v2[bx, 0:2] = 2
    v1[by, 2:4] = -2
    v2[by, 2:4] = 2
    I = np.concatenate([rows, rows], 1).reshape(-1) - 1
    J = np.concatenate([col1, col2], 1).reshape(-1) - 1
    V = np.concatenate([v1, v2], 1).reshape(-1)
    return (1.0 / (2 * h)) * sp.csr_matrix((V, (I, J)), shape=(4 * M * N, 2 * M * N))


def interior(M, N):
    """funFDNeumannBCInd.m: F and U indices (0-based) of the interior nodes."""
    k = np.arange(M * N).reshape(N, M)[1:N - 1, 1:M - 1].reshape(-1)
    iF = (4 * k[:, None] + np.arange(4)[None, :]).reshape(-1)
    iU = (2 * k[:, None] + np.arange(2)[None, :]).reshape(-1)
    return iF, iU


def subpb2_fd(M, N, h, beta, mu, U, F, udual, vdual):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    D = derivative_op(M - 2, N - 2, h)
    iF, iU = interior(M, N)
    a = (np.asarray(F) - udual)[iF]
    b = (np.asarray(U) - vdual)[iU]
    A = (beta * (D.T @ D) + mu * sp.identity(D.shape[1])).tocsc()
    out = np.array(U, np.float64, copy=True)
    out[iU] = spl.spsolve(A, beta * (D.T @ a) + mu * b)
    return out


def fd_strain(M, N, h, U):
    return derivative_op(M, N, h) @ np.asarray(U, np.float64)


def _select_beta_fd(betas, e1, e2, h):
    es = np.asarray(e1) + np.asarray(e2) * h * h
    k = int(np.argmin(es))
    if 1 <= k <= len(betas) - 2:
        p = np.polyfit(np.log10(betas[k - 1:k + 2]), es[k - 1:k + 2], 2)
        return 10 ** (-p[1] / 2 / p[0])
    return betas[k]


def frame_fd(f_raw, g_raw, winsize, step, search, tol=1e-2, mu=1e-3, n_admm=3, gridx=None,
             gridy=None, smooth=False):
    """main_ALDIC.m Sections 3-6 with the FD Subproblem 2.  gridx/gridy is
    DICpara.gridxyROIRange (funNormalizeImg statistics and the search grid);
    smooth=True adds the reference's funSmoothDisp/funSmoothStrain calls
    (main_ALDIC.m:233 on FSubpb1, :321 on FSubpb2, and in every ADMM step
    :381 on USubpb1 after its save, :400 on USubpb2, :408 on FSubpb2)."""
    import oracle as O
    f_raw, g_raw = np.asarray(f_raw), np.asarray(g_raw)
    H, W = f_raw.shape
    gx = tuple(gridx) if gridx is not None else (1, W)
    gy = tuple(gridy) if gridy is not None else (1, H)
    roi = (gx[0], gx[1], gy[0], gy[1])
    fn, _, _ = O.normalize(f_raw, roi)
    gn, mg, _ = O.normalize(g_raw, roi)
    dfdx, dfdy = O.gradient(fn)
    x, y, u, v, cc, _ = O.int_search(f_raw, g_raw, mg, gx, gy, winsize, step, (search, search))
    N, M = u.shape
    coords = np.stack([x.reshape(-1), y.reshape(-1)], 1)
    ug = O.inpaint_springs(M, N, u.reshape(-1))
    vg = O.inpaint_springs(M, N, v.reshape(-1))
    U0 = np.empty(2 * M * N)
    U0[0::2], U0[1::2] = ug, vg
    U1, F1, it, H21 = O.icgn_batch(fn, gn, dfdx, dfdy, coords, U0, winsize, tol)
    U1, F1, nbad = O.localicgn_post(M, N, it, U1, F1)
    n = M * N

    def sm(a, nf):
        return O.smooth_fields(M, N, a, nf) if smooth else a

    F1 = sm(F1, 4)
    ud, vd = np.zeros(4 * n), np.zeros(2 * n)
    betas = np.array([1e-3, np.sqrt(1e-5), 1e-2, np.sqrt(1e-3), 1e-1, np.sqrt(1e-1)]) * step * step * mu
    e1, e2 = [], []
    for b in betas:
        U2 = subpb2_fd(M, N, step, b, mu, U1, F1, ud, vd)
        F2 = fd_strain(M, N, step, U2)
        e1.append(np.linalg.norm(U1 - U2))
        e2.append(np.linalg.norm(F1 - F2))
    beta = _select_beta_fd(betas, e1, e2, step)
    U2 = subpb2_fd(M, N, step, beta, mu, U1, F1, ud, vd)
    F2 = sm(fd_strain(M, N, step, U2), 4)
    iF, iU = interior(M, N)
    ud = np.zeros(4 * n)
    vd = np.zeros(2 * n)
    ud[iF] = (F2 - F1)[iF]
    vd[iU] = (U2 - U1)[iU]
    U1old = U1.copy()
    upd, upd2 = [], []
    for _ in range(n_admm):
        U2old = U2.copy()
        U1, itb = O.subpb1_batch(fn, gn, dfdx, dfdy, coords, U2, F2, vd, H21, winsize, mu, tol)
        U1, _ = O.subpb1_post(M, N, itb, U1)
        F1 = F2.copy()
        upd2.append(np.linalg.norm(U1old - U1) / np.sqrt(2 * n))
        U1old = U1.copy()
        U1 = sm(U1, 2)
        U2 = sm(subpb2_fd(M, N, step, beta, mu, U1, F1, ud, vd), 2)
        F2 = sm(fd_strain(M, N, step, U2), 4)
        upd.append(np.linalg.norm(U2old - U2) / np.sqrt(2 * n))
        ud[iF] += (F2 - F1)[iF]
        vd[iU] += (U2 - U1)[iU]
    return dict(M=M, N=N, U=U2, F=F2, beta=beta, update_y=upd, update_y2=upd2, iters_icgn=it,
                bad_icgn=nbad)
