"""Oracle (test infrastructure only): numpy forward and backward of the
learned-initial-guess network of the library (2d_aldic_b200/csrc/cnn.cu),
used to check the GPU's outputs and gradients.  With rounding=True the bf16
roundings of the GPU path are applied at the same points (input, weights of
the tensor-core layers, every stored activation and back-propagated
activation gradient); with rounding=False everything is FP64, which the
finite-difference test uses to check this restatement's own backward pass.
The network has no counterpart in the reference.
"""
from __future__ import annotations

import numpy as np

P, PS, CELLS, C1, C2, F3, NOUT = 64, 8, 64, 128, 128, 256, 8
K = [PS * PS, C1, CELLS * CELLS, F3]
COUT = [C1, C2, F3, NOUT]
CORR_SCALE = 1.0 / np.sqrt(128.0)
TSCALE, GSCALE = 16.0, 20.0


def n_params():
    return sum(c * k + c for c, k in zip(COUT, K))


def unpack(params):
    out, o = [], 0
    for c, k in zip(COUT, K):
        W = params[o:o + c * k].reshape(c, k)
        o += c * k
        b = params[o:o + c]
        o += c
        out.append((W, b))
    return out


def bf16(x):
    """Round to the nearest bf16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def im2col(x, ps):
    """[B, H, W, C] -> rows (b, i, j), columns (di, dj, c)."""
    B, H, W, C = x.shape
    return (x.reshape(B, H // ps, ps, W // ps, ps, C).transpose(0, 1, 3, 2, 4, 5)
            .reshape(B * (H // ps) * (W // ps), ps * ps * C))


def _r(x, rounding):
    return bf16(x).astype(np.float64) if rounding else np.asarray(x, np.float64)


def forward(params, x, rounding=True):
    """Network outputs (B x 8) and the stored activations.  x: B x 64 x 64 x 2
    (reference, deformed)."""
    L = unpack(np.asarray(params, np.float64))
    B = x.shape[0]
    xin = _r(x, rounding)
    X = np.concatenate([xin[..., 0], xin[..., 1]], 0)[..., None]       # encoder batch of 2B
    Wb = [_r(W, rounding) for W, _ in L[:3]] + [np.asarray(L[3][0], np.float64)]
    cols = im2col(X, PS)
    e1 = _r(np.maximum(cols @ Wb[0].T + L[0][1], 0), rounding)
    e2 = _r(e1 @ Wb[1].T + L[1][1], rounding)
    ef = e2[:B * CELLS].reshape(B, CELLS, C2)
    eg = e2[B * CELLS:].reshape(B, CELLS, C2)
    corr = _r(CORR_SCALE * (ef @ eg.transpose(0, 2, 1)), rounding).reshape(B, CELLS * CELLS)
    y3 = _r(np.maximum(corr @ Wb[2].T + L[2][1], 0), rounding)
    out = y3 @ Wb[3].T + L[3][1]
    return out, dict(cols=cols, e1=e1, e2=e2, ef=ef, eg=eg, corr=corr, y3=y3, Wb=Wb)


def loss_grad(out, tgt):
    """The library's loss (squared error on the six warp outputs + binary
    cross-entropy of the confidence against "translation within 0.5 px") and
    d loss / d out."""
    B = out.shape[0]
    d = np.zeros_like(out)
    e = out[:, :6] - tgt
    loss = (e ** 2).sum() / B
    d[:, :6] = 2 * e / B
    err = np.maximum(np.abs(e[:, 0]), np.abs(e[:, 1])) * TSCALE
    c = (err < 0.5).astype(np.float64)
    z = out[:, 6]
    loss += (np.maximum(z, 0) - z * c + np.log1p(np.exp(-np.abs(z)))).sum() / B
    d[:, 6] = (1 / (1 + np.exp(-z)) - c) / B
    return loss, d


def backward(params, x, tgt, rounding=True):
    """(loss, packed gradients, outputs)."""
    out, A = forward(params, x, rounding)
    loss, dout = loss_grad(out, np.asarray(tgt, np.float64))
    B = x.shape[0]
    Wb = A["Wb"]
    g = [None] * 4
    y3, corr, e1, ef, eg = A["y3"], A["corr"], A["e1"], A["ef"], A["eg"]
    g[3] = (dout.T @ y3, dout.sum(0))
    dz3 = _r((dout @ Wb[3]) * (y3 > 0), rounding)
    g[2] = (dz3.T @ corr, dz3.sum(0))
    dcorr = _r(dz3 @ Wb[2], rounding).reshape(B, CELLS, CELLS)
    def_ = _r(CORR_SCALE * (dcorr @ eg), rounding)
    deg = _r(CORR_SCALE * (dcorr.transpose(0, 2, 1) @ ef), rounding)
    de2 = np.concatenate([def_.reshape(B * CELLS, C2), deg.reshape(B * CELLS, C2)])
    g[1] = (de2.T @ e1, de2.sum(0))
    dz1 = _r((de2 @ Wb[1]) * (e1 > 0), rounding)
    g[0] = (dz1.T @ A["cols"], dz1.sum(0))
    flat = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in g])
    return loss, flat, out
