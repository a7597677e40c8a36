"""Oracle (test infrastructure only): numpy forward and backward of the
learned-initial-guess network of the library (2d_aldic_b200/csrc/cnn.cu),
used to check the GPU's outputs and gradients.  With rounding=True the bf16
roundings of the GPU path are applied at the same points (input, weights of
the four tensor-core layers, every stored activation and back-propagated
activation gradient); with rounding=False everything is FP64, which the
finite-difference test uses to check this restatement's own backward pass.
The network has no counterpart in the reference.
"""
from __future__ import annotations

import numpy as np

P, CIN, C1, C2, C3, F4, NOUT = 64, 2, 64, 128, 256, 256, 8
K = [4 * 4 * CIN, 2 * 2 * C1, 2 * 2 * C2, 4 * 4 * C3, F4]
COUT = [C1, C2, C3, F4, NOUT]
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


def col2im(y, shape, ps):
    B, H, W, C = shape
    return (y.reshape(B, H // ps, W // ps, ps, ps, C).transpose(0, 1, 3, 2, 4, 5)
            .reshape(B, H, W, C))


def _r(x, rounding):
    return bf16(x).astype(np.float64) if rounding else np.asarray(x, np.float64)


def forward(params, x, rounding=True):
    """Network outputs (B x 8) and the stored activations."""
    L = unpack(np.asarray(params, np.float64))
    B = x.shape[0]
    x0 = _r(x, rounding)
    Wb = [_r(W, rounding) if l < 4 else np.asarray(W, np.float64) for l, (W, _) in enumerate(L)]
    y1 = _r(np.maximum(im2col(x0, 4) @ Wb[0].T + L[0][1], 0), rounding).reshape(B, 16, 16, C1)
    y2 = _r(np.maximum(im2col(y1, 2) @ Wb[1].T + L[1][1], 0), rounding).reshape(B, 8, 8, C2)
    y3 = _r(np.maximum(im2col(y2, 2) @ Wb[2].T + L[2][1], 0), rounding).reshape(B, 4, 4, C3)
    y4 = _r(np.maximum(y3.reshape(B, -1) @ Wb[3].T + L[3][1], 0), rounding)
    out = y4 @ Wb[4].T + L[4][1]
    return out, dict(x0=x0, y1=y1, y2=y2, y3=y3, y4=y4, Wb=Wb)


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
    L = unpack(np.asarray(params, np.float64))
    B = x.shape[0]
    Wb = A["Wb"]
    g = [None] * 5
    y4, y3, y2, y1, x0 = A["y4"], A["y3"].reshape(B, -1), A["y2"], A["y1"], A["x0"]
    g[4] = (dout.T @ y4, dout.sum(0))
    dz4 = _r((dout @ Wb[4]) * (y4 > 0), rounding)
    g[3] = (dz4.T @ y3, dz4.sum(0))
    dz3 = _r((dz4 @ Wb[3]) * (y3 > 0), rounding).reshape(B * 16, C3)
    g[2] = (dz3.T @ im2col(y2, 2), dz3.sum(0))
    dz2 = _r(col2im(dz3 @ Wb[2], y2.shape, 2) * (y2 > 0), rounding)
    dz2r = dz2.reshape(B * 64, C2)
    g[1] = (dz2r.T @ im2col(y1, 2), dz2r.sum(0))
    dz1 = _r(col2im(dz2r @ Wb[1], y1.shape, 2) * (y1 > 0), rounding)
    dz1r = dz1.reshape(B * 256, C1)
    g[0] = (dz1r.T @ im2col(x0, 4), dz1r.sum(0))
    flat = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in g])
    return loss, flat, out
