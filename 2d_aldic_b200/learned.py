"""Training and evaluation of the learned initial guess (InitNet).

Training pairs: 64 x 64 reference / deformed speckle patches (dot radius
2-4 px, seed 3) under random affine warps -- translation uniform in
+-16 px, displacement-gradient terms uniform in +-0.05 -- plus Gaussian
noise (sigma 2 grey levels) on both patches, labelled by the library's own
IC-GN started from the true warp (converged subsets only).  The pairs are
generated on the GPU as 96 x 96 tiles of two large images so that IC-GN can
run on them in one launch; the network sees the central 64 x 64 crops.

    from importlib import import_module
    L = import_module("2d_aldic_b200.learned")
    data = L.make_pairs(200_000)
    net = L.train(data, epochs=8)
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import api, synth

TILE = 96


def _affine_tiles(S, centres, t, G, noise, gen):
    """Reference and deformed 96 x 96 tiles around integer centres of the
    speckle image S (float64 (H, W)); the deformed tile is S at
    X = c + (I + G)^-1 (x - c - t) (bicubic, clamp to edge)."""
    import torch
    dev = S.device
    q = torch.arange(TILE, device=dev, dtype=torch.float64) - TILE // 2
    qy, qx = torch.meshgrid(q, q, indexing="ij")                     # tile row = y
    n = centres.shape[0]
    cx = centres[:, 0].view(n, 1, 1)
    cy = centres[:, 1].view(n, 1, 1)
    H, W = S.shape
    xs = (cx + qx).long().clamp(1, W) - 1
    ys = (cy + qy).long().clamp(1, H) - 1
    F = S[ys, xs]
    a, b, c, d = 1 + G[:, 0], G[:, 2], G[:, 1], 1 + G[:, 3]           # [[1+ux, uy], [vx, 1+vy]]
    det = a * d - b * c
    ia, ib, ic, id_ = d / det, -b / det, -c / det, a / det
    rx = qx - t[:, 0].view(n, 1, 1)
    ry = qy - t[:, 1].view(n, 1, 1)
    X = cx + ia.view(n, 1, 1) * rx + ib.view(n, 1, 1) * ry
    Y = cy + ic.view(n, 1, 1) * rx + id_.view(n, 1, 1) * ry
    Gt = synth.bicubic_sample_t(S, X, Y)
    F = F + noise * torch.randn(F.shape, generator=gen, dtype=torch.float64, device=dev)
    Gt = Gt + noise * torch.randn(Gt.shape, generator=gen, dtype=torch.float64, device=dev)
    return F, Gt


def make_pairs(n: int, seed: int = 3, device: int = 0, chunk: int = 8192, noise: float = 2.0,
               tmax: float = 16.0, gmax: float = 0.05, label_tol: float = 1e-3, log=None):
    """n labelled training pairs on the GPU: dict with x (n' x 64 x 64 x 2
    bf16), targets (n' x 6 FP32, the network's output scaling), truth (n' x 6:
    u, v, F11, F21, F12, F22 of the generating warp), kept n' <= n (IC-GN
    converged)."""
    import torch
    dev = torch.device("cuda", device)
    rng = np.random.Generator(np.random.PCG64(seed))
    side = 4096
    S = synth.speckle_t(side, side, 520_000, seed, device=dev)
    gen = torch.Generator(device=dev).manual_seed(seed + 1000)
    ctx = api.Context(device)
    xs, tg, tr = [], [], []
    for s0 in range(0, n, chunk):
        m = min(chunk, n - s0)
        cen = rng.integers(TILE, side - TILE, (m, 2)).astype(np.float64)
        t = rng.uniform(-tmax, tmax, (m, 2))
        G = rng.uniform(-gmax, gmax, (m, 4))              # [ux, vx, uy, vy] = [F11 F21 F12 F22]
        tc = lambda a: torch.as_tensor(a, device=dev)
        F, Gt = _affine_tiles(S, tc(cen), tc(t), tc(G), noise, gen)
        T = int(math.ceil(math.sqrt(m)))
        big = lambda tl: (torch.zeros((T * T, TILE, TILE), dtype=torch.float64, device=dev)
                          .index_copy_(0, torch.arange(m, device=dev), tl)
                          .view(T, T, TILE, TILE).permute(0, 2, 1, 3).reshape(T * TILE, T * TILE)
                          .to(torch.float32).contiguous())
        Fb, Gb = big(F), big(Gt)
        k = np.arange(m)
        coords = np.stack([(k % T) * TILE + TILE // 2 + 1, (k // T) * TILE + TILE // 2 + 1], 1).astype(np.float64)
        ctx.set_ref(Fb)
        ctx.set_def(Gb)
        U0 = np.empty(2 * m)
        U0[0::2], U0[1::2] = t[:, 0], t[:, 1]
        U, Fo, it, _ = api.local_icgn(ctx, coords, U0, 32, label_tol, api.FP32)
        ok = (it >= 1) & (it <= 100) & np.isfinite(U[0::2]) & np.isfinite(U[1::2])
        if log:
            e = np.hypot(U[0::2] - t[:, 0], U[1::2] - t[:, 1])
            log(f"pairs {s0}..{s0 + m}: {ok.mean():.3f} converged, label - truth median "
                f"{np.median(e[ok]) if ok.any() else float('nan'):.4f} px, max "
                f"{e[ok].max() if ok.any() else float('nan'):.3f} px")
        x = api.cnn_patches(ctx, coords[ok], bf16=True)
        tgt = np.concatenate([U.reshape(-1, 2)[ok] / InitScale.T, Fo.reshape(-1, 4)[ok] * InitScale.G], 1)
        xs.append(x)
        tg.append(torch.as_tensor(tgt, dtype=torch.float32, device=dev))
        tr.append(np.concatenate([t, G], 1)[ok])
        del F, Gt, Fb, Gb
    ctx.close()
    return {"x": torch.cat(xs), "targets": torch.cat(tg), "truth": np.concatenate(tr)}


class InitScale:
    T = api.InitNet.TSCALE
    G = api.InitNet.GSCALE


def train(data, epochs: int = 8, batch: int = 256, lr: float = 1e-3, seed: int = 0, device: int = 0,
          net: api.InitNet | None = None, log=None):
    """Adam with a cosine learning-rate decay over the epochs; returns the net."""
    import torch
    net = net or api.InitNet(device, seed)
    x, t = data["x"], data["targets"]
    n = x.shape[0]
    g = torch.Generator(device=x.device).manual_seed(seed)
    steps = epochs * (n // batch)
    k = 0
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g, device=x.device)
        tot = 0.0
        for b in range(n // batch):
            idx = perm[b * batch:(b + 1) * batch]
            a = lr * 0.5 * (1 + math.cos(math.pi * k / max(1, steps)))
            loss, _, _ = net.train_step(x[idx], t[idx], a)
            tot += loss
            k += 1
        if log:
            log(f"epoch {ep + 1}/{epochs} loss {tot / max(1, n // batch):.5f} "
                f"({time.perf_counter() - t0:.1f} s)")
    return net


def evaluate(net: api.InitNet, data, batch: int = 4096):
    """Translation error of the network against the IC-GN labels (px)."""
    import torch
    x, t = data["x"], data["targets"]
    outs = [net.predict(x[b:b + batch]) for b in range(0, x.shape[0], batch)]
    o = torch.cat(outs).cpu().numpy()
    tt = t.cpu().numpy()
    e = (o[:, :2] - tt[:, :2]) * InitScale.T
    r = np.sqrt((e ** 2).sum(1))
    eg = (o[:, 2:6] - tt[:, 2:6]) / InitScale.G
    conf = 1 / (1 + np.exp(-o[:, 6]))
    return {"rms_px": float(np.sqrt((r ** 2).mean())), "median_px": float(np.median(r)),
            "within_0.5px": float((r < 0.5).mean()), "within_1px": float((r < 1).mean()),
            "rms_gradient": float(np.sqrt((eg ** 2).mean())),
            "confident": float((conf > 0.5).mean()),
            "within_0.5px_when_confident": float((r[conf > 0.5] < 0.5).mean()) if (conf > 0.5).any() else None}
