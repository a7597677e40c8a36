"""The finite-difference Subproblem 2 (funDerivativeOp.m and the FD branch of
main_ALDIC.m): the oracle's vectorised operator against a literal
transcription of funDerivativeOp's per-node loop, and its properties.  CPU
only."""
import numpy as np

from oracle import fd as FD


def _literal(M, N, h):
    """funDerivativeOp.m:12-44, node by node (1-based indices as written)."""
    A = np.zeros((4 * M * N, 2 * M * N))
    for tempi in range(M * N):
        tx, ty = tempi % M + 1, tempi // M + 1
        border = [1, 1, 1, 1]
        if ty == 1: border[1] = 0
        if ty == N: border[0] = 0
        if tx == 1: border[3] = 0
        if tx == M: border[2] = 0
        index = tx + M * (ty - 1)
        nb = [index + b * o for b, o in zip(border, [M, -M, 1, -1])]
        rows = [4 * index - 3, 4 * index - 2, 4 * index - 1, 4 * index]
        col1 = [2 * nb[3] - 1, 2 * nb[3], 2 * nb[1] - 1, 2 * nb[1]]
        col2 = [2 * nb[2] - 1, 2 * nb[2], 2 * nb[0] - 1, 2 * nb[0]]
        val = [-1.0] * 4 + [1.0] * 4
        if border[2] * border[3] == 0:
            val[0] = val[1] = -2.0
            val[4] = val[5] = 2.0
        if border[0] * border[1] == 0:
            val[2] = val[3] = -2.0
            val[6] = val[7] = 2.0
        for r, c, v in zip(rows + rows, col1 + col2, val):
            A[r - 1, c - 1] += v
    return A / (2 * h)


def test_derivative_op_matches_literal():
    for M, N in [(5, 4), (7, 6), (3, 3)]:
        np.testing.assert_array_equal(FD.derivative_op(M, N, 8.0).toarray(), _literal(M, N, 8.0))


def test_derivative_op_exact_on_affine_fields():
    M, N, h = 9, 7, 10.0
    k = np.arange(M * N)
    x, y = h * (k % M), h * (k // M)
    U = np.empty(2 * M * N)
    U[0::2] = 0.3 + 0.01 * x - 0.02 * y
    U[1::2] = -1.0 + 0.005 * x + 0.03 * y
    F = FD.fd_strain(M, N, h, U).reshape(-1, 4)
    np.testing.assert_allclose(F, np.tile([0.01, 0.005, -0.02, 0.03], (M * N, 1)), atol=1e-14)


def test_subpb2_fd_consistent_data_is_a_fixed_point():
    """With F = D2 U of an affine field and zero duals the interior solution
    is U itself (D'D U = D'F, mass term consistent)."""
    M, N, h = 8, 6, 16.0
    k = np.arange(M * N)
    x, y = h * (k % M), h * (k // M)
    U = np.empty(2 * M * N)
    U[0::2] = 1.0 + 0.002 * x
    U[1::2] = -0.5 + 0.004 * y - 0.001 * x
    F = FD.fd_strain(M, N, h, U)
    out = FD.subpb2_fd(M, N, h, 0.05, 1e-3, U, F, np.zeros(4 * M * N), np.zeros(2 * M * N))
    np.testing.assert_allclose(out, U, atol=1e-9)
