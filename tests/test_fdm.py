"""The direct Subproblem 2 solver's building blocks on the CPU (no device
work): the 1-D eigenbases the library computes on the host for the fast
diagonalisation of the uniform-mesh operators (aldic_fdm_basis), and the
Kronecker-sum identity the solver rests on, checked against the reference's
own assembly rules:

* FE: Subpb2.m's element loop (the scipy restatement in test_oracle.py)
  equals beta (Kx (x) My + Mx (x) Ky) + mu Mx (x) My per displacement
  component, K and M the 1-D linear-element stiffness and mass;
* FD: funDerivativeOp's (beta D'D + mu I) on the interior grid (oracle/fd.py)
  equals beta (I (x) Gx + Gy (x) I) + mu I, G = d'd of the 1-D difference.

The solution through the library's bases then matches the sparse direct
solve to 1e-10 relative.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sl
import scipy.sparse.linalg as spla

from oracle import fd as FD
from test_oracle import subpb2_system

FDM_FE, FDM_FD = 0, 1


def basis(aldic, t, n, h):
    V = np.empty((n, n))
    lam = np.empty(n)
    rc = aldic._lib.lib().aldic_fdm_basis(t, n, C.c_double(h), V.ctypes.data_as(C.c_void_p),
                                          lam.ctypes.data_as(C.c_void_p))
    assert rc == 0
    return V, lam


def fe_1d(n, h):
    K = np.zeros((n, n))
    Mm = np.zeros((n, n))
    for e in range(n - 1):
        K[e:e + 2, e:e + 2] += np.array([[1.0, -1.0], [-1.0, 1.0]]) / h
        Mm[e:e + 2, e:e + 2] += np.array([[2.0, 1.0], [1.0, 2.0]]) * h / 6
    return K, Mm


def fd_1d(n, h):
    """d'd of funDerivativeOp.m along one line (central / 2h, one-sided and
    doubled at the ends), from the oracle's 2-D operator on an n x 1 grid."""
    D = FD.derivative_op(n, 1, h).toarray()      # rows F11 F21 F12 F22, columns u v
    dx = D[0::4, 0::2]                           # du/dx rows, u columns
    return dx.T @ dx


@pytest.mark.parametrize("n", [2, 3, 7, 64, 243])
@pytest.mark.parametrize("h", [4.0, 16.0])
def test_basis_fe(aldic, n, h):
    V, lam = basis(aldic, FDM_FE, n, h)
    K, Mm = fe_1d(n, h)
    np.testing.assert_allclose(V.T @ Mm @ V, np.eye(n), atol=1e-13)
    np.testing.assert_allclose(V.T @ K @ V, np.diag(lam), atol=1e-13 / h)
    np.testing.assert_allclose(np.sort(lam), sl.eigh(K, Mm, eigvals_only=True), atol=1e-13 / h)


@pytest.mark.parametrize("n", [2, 3, 7, 64, 241])
@pytest.mark.parametrize("h", [4.0, 16.0])
def test_basis_fd(aldic, n, h):
    V, lam = basis(aldic, FDM_FD, n, h)
    G = fd_1d(n, h)
    np.testing.assert_allclose(V.T @ V, np.eye(n), atol=1e-13)
    np.testing.assert_allclose(V.T @ G @ V, np.diag(lam), atol=1e-14)
    np.testing.assert_allclose(np.sort(lam), np.linalg.eigvalsh(G), atol=1e-14)


def fdm_apply_inverse(Vx, lx, Vy, ly, beta, mu, B):
    """X = Vy ((Vy' B Vx) ./ D) Vx' for a field B (N x M, x fastest)."""
    Cm = Vy.T @ B @ Vx
    Cm /= beta * (ly[:, None] + lx[None, :]) + mu
    return Vy @ Cm @ Vx.T


@pytest.mark.parametrize("M,N", [(9, 7), (16, 23)])
def test_fe_operator_is_the_kronecker_sum(aldic, M, N):
    rng = np.random.default_rng(3)
    h, mu = 8.0, 1e-3
    n = M * N
    U = rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    ud = 0.001 * rng.standard_normal(4 * n)
    vd = 0.01 * rng.standard_normal(2 * n)
    Vx, lx = basis(aldic, FDM_FE, M, h)
    Vy, ly = basis(aldic, FDM_FE, N, h)
    Kx, Mx = fe_1d(M, h)
    Ky, My = fe_1d(N, h)
    for beta in (1e-3 * h * h * mu, 0.1 * h * h * mu):
        A, b = subpb2_system(M, N, h, beta, mu, U, F, ud, vd)
        # per component, node order x fastest: slow index y, fast index x
        Ak = beta * (np.kron(My, Kx) + np.kron(Ky, Mx)) + mu * np.kron(My, Mx)
        Ad = A.toarray()
        np.testing.assert_allclose(Ad[0::2, 0::2], Ak, atol=1e-15, rtol=1e-12)
        np.testing.assert_allclose(Ad[1::2, 1::2], Ak, atol=1e-15, rtol=1e-12)
        assert np.abs(Ad[0::2, 1::2]).max() == 0.0
        ref = spla.spsolve(A.tocsc(), b)
        for f in (0, 1):
            X = fdm_apply_inverse(Vx, lx, Vy, ly, beta, mu, b[f::2].reshape(N, M))
            np.testing.assert_allclose(X.reshape(-1), ref[f::2], rtol=1e-10,
                                       atol=1e-10 * np.abs(ref).max())


@pytest.mark.parametrize("M,N", [(9, 7), (14, 20)])
def test_fd_operator_is_the_kronecker_sum(aldic, M, N):
    rng = np.random.default_rng(4)
    h, mu = 10.0, 1e-3
    n = M * N
    U = rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    ud = 0.001 * rng.standard_normal(4 * n)
    vd = 0.01 * rng.standard_normal(2 * n)
    Mi, Ni = M - 2, N - 2
    Vx, lx = basis(aldic, FDM_FD, Mi, h)
    Vy, ly = basis(aldic, FDM_FD, Ni, h)
    D = FD.derivative_op(Mi, Ni, h)
    Gx, Gy = fd_1d(Mi, h), fd_1d(Ni, h)
    DtD = (D.T @ D).toarray()
    Gk = np.kron(np.eye(Ni), Gx) + np.kron(Gy, np.eye(Mi))
    np.testing.assert_allclose(DtD[0::2, 0::2], Gk, atol=1e-15)
    np.testing.assert_allclose(DtD[1::2, 1::2], Gk, atol=1e-15)
    for beta in (1e-3 * h * h * mu, 0.3 * h * h * mu):
        ref = FD.subpb2_fd(M, N, h, beta, mu, U, F, ud, vd)
        iF, iU = FD.interior(M, N)
        a = (F - ud)[iF]
        bb = (U - vd)[iU]
        rhs = beta * (D.T @ a) + mu * bb
        for f in (0, 1):
            X = fdm_apply_inverse(Vx, lx, Vy, ly, beta, mu, rhs[f::2].reshape(Ni, Mi))
            np.testing.assert_allclose(X.reshape(-1), ref[iU][f::2], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("M,N", [(9, 7), (16, 23)])
def test_fe_beta_sweep_from_the_right_hand_side_parts(aldic, M, N):
    """The identity fdm_solve_sweep rests on: the Subpb2 right-hand side is
    beta b(1, 0) + mu b(0, 1), so transforming the two parts once and forming
    (beta C_beta + mu C_mu) / (beta (ly + lx) + mu) in the eigen domain gives
    each of the sweep's six systems' solutions."""
    rng = np.random.default_rng(5)
    h, mu = 8.0, 1e-3
    n = M * N
    U = rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    ud = 0.001 * rng.standard_normal(4 * n)
    vd = 0.01 * rng.standard_normal(2 * n)
    Vx, lx = basis(aldic, FDM_FE, M, h)
    Vy, ly = basis(aldic, FDM_FE, N, h)
    _, b_beta = subpb2_system(M, N, h, 1.0, 0.0, U, F, ud, vd)
    _, b_mu = subpb2_system(M, N, h, 0.0, 1.0, U, F, ud, vd)
    lam = ly[:, None] + lx[None, :]
    base = h * h * mu
    for k, scale in enumerate((1e-3, 1e-5 ** 0.5, 1e-2, 1e-3 ** 0.5, 1e-1, 1e-1 ** 0.5)):
        beta = scale * base
        A, b = subpb2_system(M, N, h, beta, mu, U, F, ud, vd)
        np.testing.assert_allclose(b, beta * b_beta + mu * b_mu, rtol=1e-12,
                                   atol=1e-14 * np.abs(b).max())
        ref = spla.spsolve(A.tocsc(), b)
        for f in (0, 1):
            Cb = Vy.T @ b_beta[f::2].reshape(N, M) @ Vx
            Cm = Vy.T @ b_mu[f::2].reshape(N, M) @ Vx
            X = Vy @ ((beta * Cb + mu * Cm) / (beta * lam + mu)) @ Vx.T
            np.testing.assert_allclose(X.reshape(-1), ref[f::2], rtol=1e-10,
                                       atol=1e-10 * np.abs(ref).max())
