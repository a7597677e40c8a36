"""The BF16 tcgen05 GEMM of the learned initial guess against a PyTorch FP32
reference of the same product (inputs rounded to bf16 first, so only the
accumulation order differs): plain, ragged, bias/ReLU/bf16 epilogue, several
N tiles, transposed and patch (im2col) operands, patch scatter with a ReLU
mask, split-K, and batches of scaled products."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(aldic):
    import torch
    assert torch.cuda.is_available()
    return aldic, aldic.Context(0), torch


def _op(L, t, mode, rows, kdim, ld=0, geo=(0, 0, 0, 0), bstride=0):
    o = L.GemmOperand()
    o.p, o.ld, o.mode, o.rows, o.kdim, o.bstride = t.data_ptr(), ld, mode, rows, kdim, bstride
    o.Hin, o.Win, o.C, o.ps = geo
    return o


def _out(L, t, M, N, ld=0, fp32=1, bias=None, relu=0, mode=0, mask=None, geo=(0, 0, 0, 0),
         split_stride=0, scale=1.0, bstride=0):
    d = L.GemmOutput()
    d.p, d.ld, d.mode, d.fp32 = t.data_ptr(), ld, mode, fp32
    d.bias = bias.data_ptr() if bias is not None else None
    d.relu = relu
    d.mask = mask.data_ptr() if mask is not None else None
    d.Hin, d.Win, d.C, d.ps = geo
    d.M, d.N, d.split_stride, d.scale, d.bstride = M, N, split_stride, scale, bstride
    return d


def _gemm(env, A, B, D, splits=1, batches=1):
    aldic, ctx, torch = env
    aldic._lib.call("aldic_gemm_bf16", ctx.h, C.byref(A), C.byref(B), C.byref(D), splits, batches)
    torch.cuda.synchronize()


def _rand(torch, *shape, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return (torch.randn(*shape, generator=g, device="cuda") * 0.5).to(torch.bfloat16)


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (300, 40, 200), (1024, 256, 1024),
                                   (256, 512, 4096), (2000, 128, 72)])
def test_gemm_rows(env, M, N, K):
    aldic, ctx, torch = env
    L = aldic._lib
    A = _rand(torch, M, K, seed=1)
    B = _rand(torch, N, K, seed=2)
    D = torch.full((M, N), float("nan"), device="cuda")
    _gemm(env, _op(L, A, 0, M, K, K), _op(L, B, 0, N, K, K), _out(L, D, M, N, N))
    ref = A.float() @ B.float().T
    torch.testing.assert_close(D, ref, rtol=1e-4, atol=1e-4 * K ** 0.5)


def test_gemm_bias_relu_bf16(env):
    aldic, ctx, torch = env
    L = aldic._lib
    M, N, K = 512, 128, 256
    A, B = _rand(torch, M, K, seed=3), _rand(torch, N, K, seed=4)
    bias = torch.randn(N, device="cuda")
    D = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    _gemm(env, _op(L, A, 0, M, K, K), _op(L, B, 0, N, K, K),
          _out(L, D, M, N, N, fp32=0, bias=bias, relu=1))
    ref = torch.relu(A.float() @ B.float().T + bias)
    torch.testing.assert_close(D.float(), ref, rtol=1e-2, atol=2e-2)


def test_gemm_transposed_operands(env):
    aldic, ctx, torch = env
    L = aldic._lib
    M, N, K = 264, 96, 320
    At = _rand(torch, K, M, seed=5)          # A = At^T
    Bt = _rand(torch, K, N, seed=6)          # B = Bt^T
    D = torch.empty((M, N), device="cuda")
    _gemm(env, _op(L, At, 2, M, K, M), _op(L, Bt, 2, N, K, N), _out(L, D, M, N, N))
    ref = At.float().T @ Bt.float()
    torch.testing.assert_close(D, ref, rtol=1e-4, atol=1e-3)


def _im2col(torch, X, ps):
    Bn, H, W, Cc = X.shape
    return (X.view(Bn, H // ps, ps, W // ps, ps, Cc).permute(0, 1, 3, 2, 4, 5)
            .reshape(Bn * (H // ps) * (W // ps), ps * ps * Cc))


def _col2im(torch, Y, shape, ps):
    Bn, H, W, Cc = shape
    return (Y.view(Bn, H // ps, W // ps, ps, ps, Cc).permute(0, 1, 3, 2, 4, 5)
            .reshape(Bn, H, W, Cc))


def test_gemm_patch_forward_and_backward(env):
    aldic, ctx, torch = env
    L = aldic._lib
    Bn, H, W, Cin, ps, Cout = 3, 16, 16, 8, 4, 16
    geo = (H, W, Cin, ps)
    X = _rand(torch, Bn, H, W, Cin, seed=7)
    Wt = _rand(torch, Cout, ps * ps * Cin, seed=8)
    M, K = Bn * (H // ps) * (W // ps), ps * ps * Cin
    cols = _im2col(torch, X, ps).float()
    # forward: Y = im2col(X) . W^T
    Y = torch.empty((M, Cout), device="cuda")
    _gemm(env, _op(L, X, 1, M, K, geo=geo), _op(L, Wt, 0, Cout, K, K), _out(L, Y, M, Cout, Cout))
    torch.testing.assert_close(Y, cols @ Wt.float().T, rtol=1e-4, atol=1e-3)
    # weight gradient: dW = dZ^T . im2col(X)   (A transposed rows, B transposed patches)
    dZ = _rand(torch, M, Cout, seed=9)
    dW = torch.empty((Cout, K), device="cuda")
    _gemm(env, _op(L, dZ, 2, Cout, M, Cout), _op(L, X, 3, K, M, geo=geo), _out(L, dW, Cout, K, K))
    torch.testing.assert_close(dW, dZ.float().T @ cols, rtol=1e-4, atol=1e-3)
    # input gradient: dX = col2im(dZ . W), masked by a ReLU pattern
    mask = _rand(torch, Bn, H, W, Cin, seed=10)
    dX = torch.full((Bn, H, W, Cin), 7.0, dtype=torch.bfloat16, device="cuda")
    _gemm(env, _op(L, dZ, 0, M, Cout, Cout), _op(L, Wt, 2, K, Cout, K),
          _out(L, dX, M, K, fp32=0, mode=1, mask=mask, geo=geo))
    ref = _col2im(torch, dZ.float() @ Wt.float(), (Bn, H, W, Cin), ps) * (mask.float() > 0)
    torch.testing.assert_close(dX.float(), ref, rtol=1e-2, atol=2e-2)


def test_gemm_split_k(env):
    aldic, ctx, torch = env
    L = aldic._lib
    M, N, K, S = 256, 64, 2048, 4
    A, B = _rand(torch, M, K, seed=11), _rand(torch, N, K, seed=12)
    P = torch.empty((S, M, N), device="cuda")
    _gemm(env, _op(L, A, 0, M, K, K), _op(L, B, 0, N, K, K),
          _out(L, P, M, N, N, split_stride=M * N), splits=S)
    torch.testing.assert_close(P.sum(0), A.float() @ B.float().T, rtol=1e-4, atol=1e-3)


def test_gemm_rejects_misaligned(env):
    aldic, ctx, torch = env
    L = aldic._lib
    A = _rand(torch, 128, 72, seed=13)
    D = torch.empty((128, 64), device="cuda")
    with pytest.raises(aldic.AldicError):
        _gemm(env, _op(L, A, 0, 128, 70, 70), _op(L, A, 0, 64, 70, 70), _out(L, D, 128, 64, 64))


def test_gemm_batched_scaled(env):
    aldic, ctx, torch = env
    L = aldic._lib
    nb, M, N, K = 37, 64, 64, 128
    A = _rand(torch, nb, M, K, seed=14)
    B = _rand(torch, nb, N, K, seed=15)
    D = torch.empty((nb, M, N), device="cuda")
    _gemm(env, _op(L, A, 0, M, K, K, bstride=M * K), _op(L, B, 0, N, K, K, bstride=N * K),
          _out(L, D, M, N, N, scale=0.125, bstride=M * N), batches=nb)
    ref = torch.bmm(A.float(), B.float().transpose(1, 2)) * 0.125
    torch.testing.assert_close(D, ref, rtol=1e-4, atol=1e-4)
    # transposed operands inside a batch (the correlation's backward products)
    At = _rand(torch, nb, K, M, seed=16)
    D2 = torch.empty((nb, M, N), device="cuda")
    _gemm(env, _op(L, At, 2, M, K, M, bstride=M * K), _op(L, B, 0, N, K, K, bstride=N * K),
          _out(L, D2, M, N, N, bstride=M * N), batches=nb)
    torch.testing.assert_close(D2, torch.bmm(At.float().transpose(1, 2), B.float().transpose(1, 2)),
                               rtol=1e-4, atol=1e-4)
