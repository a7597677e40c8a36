"""Oracle (test infrastructure only): numpy restatement of ComputeStrain.m
(main_ALDIC.m Section 8) on the uniform mesh, for tests/: methods 0 (solved
F), 1 (funDerivativeOp), 2 (PlaneFit2.m, solved per node by its normal
equations as written), 3 (funGlobal_NodalStrainAvg, the C oracle), and the
strain types of ComputeStrain.m:105-129."""
from __future__ import annotations

import numpy as np


def plane_fit2(Ug, hx, hy, rad):
    """plotFiles/PlaneFit2.m: per interior node the least-squares plane over
    the (2 rad + 1)^2 window; Ug is M x N (first index x).  Returns UY, UX."""
    M, N = Ug.shape
    UY, UX = Ug.copy(), Ug.copy()
    A = np.array([[1.0, ti * hx, tj * hy] for tj in range(-rad, rad + 1) for ti in range(-rad, rad + 1)])
    for ii in range(rad, M - rad):
        for jj in range(rad, N - rad):
            b = np.array([Ug[ii + ti, jj + tj] for tj in range(-rad, rad + 1) for ti in range(-rad, rad + 1)])
            v = np.linalg.solve(A.T @ A, A.T @ b)
            UX[ii, jj], UY[ii, jj] = v[1], v[2]
    return UY, UX


def compute_strain(M, N, h, method, rad, stype, U=None, F=None):
    import oracle as O
    from oracle import fd as FD
    if method == 0:
        fs = np.array(F, np.float64, copy=True)
    elif method == 3:
        fs = O.nodal_strain(M, N, h, U)
    else:
        fs = FD.fd_strain(M, N, h, U)
        if method == 2:
            u = np.asarray(U)[0::2].reshape(N, M).T          # reshape(U(1:2:end), M, N)
            v = np.asarray(U)[1::2].reshape(N, M).T
            uy, ux = plane_fit2(u, h, h, rad)
            vy, vx = plane_fit2(v, h, h, rad)
            g = fs.reshape(N, M, 4)
            sl = (slice(rad, N - rad), slice(rad, M - rad))
            g[sl + (0,)] = ux.T[sl]
            g[sl + (1,)] = vx.T[sl]
            g[sl + (2,)] = uy.T[sl]
            g[sl + (3,)] = vy.T[sl]
            fs = g.reshape(-1)
    f = fs.reshape(-1, 4)
    ux, vx, uy, vy = f[:, 0], f[:, 1], f[:, 2], f[:, 3]
    out = f.copy()
    if stype == 1:
        out[:, 0] = 1 / (1 - ux) - 1
        out[:, 3] = 1 / (1 - vy) - 1
        out[:, 2] = uy / (1 - vy)
        out[:, 1] = vx / (1 - ux)
    elif stype == 2:
        out[:, 0] = 0.5 * (ux * 2 - ux ** 2 - vx ** 2)
        out[:, 3] = 0.5 * (vy * 2 - uy ** 2 - vy ** 2)
        out[:, 2] = 0.5 * (uy + vx - ux * uy - vx * vy)
        out[:, 1] = 0.5 * (vx + uy - uy * ux - vy * vx)
    return fs, out.reshape(-1)
