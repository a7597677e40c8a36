"""Seeded synthetic speckle workloads (the reference ships no generator).

Images follow the reference's layout after ReadImage's transpose: a W x H
image Img(x, y) with x the image column, stored x-fastest, i.e. a numpy array
of shape (H, W).  Pixel coordinates are 1-based like MATLAB's.

Recipe (identical for every workload):
  * RNG numpy Generator(PCG64(seed)); draw order: centres x ~ U[0,W),
    y ~ U[0,H); radii r ~ U[2,4]; peaks A ~ U[80,200];
  * dot profile A*exp(-d^2/r^2), summed, plus the background, clipped and
    quantised to the integer type;
  * deformed image: the reference sampled (Keys bicubic, clamp-to-edge) at
    X = x - u(X), solved by fixed-point iteration to 1e-10 px, plus N(0,s^2)
    noise from seed+1000, clipped and quantised;
  * ground truth is u(X) at node X in reference coordinates (the Lagrangian
    convention funICGN tracks: f(X) <-> g(X + u)).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable

import numpy as np

Field = Callable[[np.ndarray, np.ndarray], tuple[np.ndarray, np.ndarray]]


def speckle(W: int, H: int, ndots: int, seed: int, bg: float = 20.0,
            amp=(80.0, 200.0), radius=(2.0, 4.0), dtype=np.uint8,
            scale: float = 1.0) -> np.ndarray:
    """Gaussian-dot speckle image of shape (H, W)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cx = rng.uniform(0, W, ndots)
    cy = rng.uniform(0, H, ndots)
    r = rng.uniform(radius[0], radius[1], ndots)
    A = rng.uniform(amp[0], amp[1], ndots)
    img = np.zeros(H * W, np.float64)
    R = 12  # exp(-(12/4)^2) ~ 1.2e-4 of the peak: negligible after quantisation
    off = np.arange(-R, R + 1)
    chunk = 4096
    for s in range(0, ndots, chunk):
        e = min(ndots, s + chunk)
        px = np.floor(cx[s:e]).astype(np.int64)[:, None, None] + off[None, None, :]
        py = np.floor(cy[s:e]).astype(np.int64)[:, None, None] + off[None, :, None]
        # pixel centres at integer 0-based positions
        d2 = (px - cx[s:e, None, None]) ** 2 + (py - cy[s:e, None, None]) ** 2
        val = A[s:e, None, None] * np.exp(-d2 / (r[s:e, None, None] ** 2))
        ok = (px >= 0) & (px < W) & (py >= 0) & (py < H)
        idx = (py * W + px)[ok]
        img += np.bincount(idx, weights=val[ok], minlength=H * W)
    img = img.reshape(H, W) + bg
    img *= scale
    info = np.iinfo(dtype)
    return np.clip(np.rint(img), info.min, info.max).astype(dtype)


def keys_weights(t: np.ndarray):
    t2 = t * t
    t3 = t2 * t
    return (0.5 * (-t + 2 * t2 - t3), 0.5 * (2 - 5 * t2 + 3 * t3),
            0.5 * (t + 4 * t2 - 3 * t3), 0.5 * (-t2 + t3))


def bicubic_sample(img: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Keys bicubic (a=-1/2), clamp-to-edge, at 1-based (x, y)."""
    H, W = img.shape
    im = img.astype(np.float64)
    xf = np.floor(x)
    yf = np.floor(y)
    wx = keys_weights(x - xf)
    wy = keys_weights(y - yf)
    xi = xf.astype(np.int64) - 1  # 0-based index of floor(x)
    yi = yf.astype(np.int64) - 1
    out = np.zeros(x.shape, np.float64)
    for a in range(4):
        rows = np.clip(yi - 1 + a, 0, H - 1)
        acc = np.zeros(x.shape, np.float64)
        for b in range(4):
            cols = np.clip(xi - 1 + b, 0, W - 1)
            acc += wx[b] * im[rows, cols]
        out += wy[a] * acc
    return out


def warp(ref: np.ndarray, field: Field, noise: float, seed: int,
         dtype=None) -> np.ndarray:
    """Deformed image g(x) = f(X) + noise with x = X + u(X)."""
    H, W = ref.shape
    yy, xx = np.meshgrid(np.arange(1, H + 1, dtype=np.float64),
                         np.arange(1, W + 1, dtype=np.float64), indexing="ij")
    X, Y = xx.copy(), yy.copy()
    for _ in range(200):
        u, v = field(X, Y)
        Xn, Yn = xx - u, yy - v
        err = max(np.abs(Xn - X).max(), np.abs(Yn - Y).max())
        X, Y = Xn, Yn
        if err < 1e-10:
            break
    g = bicubic_sample(ref, X, Y)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    g = g + rng.normal(0.0, noise, g.shape)
    dtype = dtype or ref.dtype
    info = np.iinfo(dtype)
    return np.clip(np.rint(g), info.min, info.max).astype(dtype)


# ------------------------------------------------------------------ workloads
@dataclasses.dataclass
class Workload:
    name: str
    W: int
    H: int
    ndots: int
    seed: int
    winsize: int
    step: int
    search: int
    noise: float
    field: Field
    tol: float = 1e-2
    n_admm: int = 3
    fp64: bool = False
    dtype: type = np.uint8
    scale: float = 1.0

    def images(self):
        f = speckle(self.W, self.H, self.ndots, self.seed, dtype=self.dtype,
                    scale=self.scale)
        g = warp(f, self.field, self.noise * self.scale, self.seed)
        return f, g


def _affine_small(X, Y):
    return 0.5 + 0.01 * X, -0.3 + 0.005 * Y


def _sine(X, Y):
    return 2.0 * np.sin(2 * np.pi * Y / 256.0), 1.5 * np.cos(2 * np.pi * X / 256.0)


def plate_hole(cx=1024.0, cy=1024.0, rad=300.0):
    def f(X, Y):
        dx, dy = X - cx, Y - cy
        r2 = np.maximum(dx * dx + dy * dy, 1e-12)
        inside = r2 < rad * rad
        u = np.where(inside, 0.0, 0.002 * dx * (1.0 + rad * rad / r2))
        v = np.where(inside, 0.0, -0.0006 * dy)
        return u, v
    return f


def uniform_affine(ux, vy, u0=0.0, v0=0.0):
    def f(X, Y):
        return u0 + ux * X + 0.0 * Y, v0 + vy * Y + 0.0 * X
    return f


WORKLOADS = {
    # plain ALDIC, 512^2, 8000 dots, subset 20 / step 10, search +-20, FP64
    "plain512": Workload("plain512", 512, 512, 8000, 0, 20, 10, 20, 2.0, _affine_small,
                         tol=1e-3, fp64=True),
    # large uniform batch, 2048^2, 130k dots, subset 32 / step 8, sinusoidal
    "uniform2048": Workload("uniform2048", 2048, 2048, 130_000, 1, 32, 8, 16, 2.0, _sine),
}


def workload(name: str, scale_down: int = 1) -> Workload:
    """A named workload; scale_down > 1 shrinks the image (same density) for
    quick parity runs."""
    w = dataclasses.replace(WORKLOADS[name])
    if scale_down > 1:
        w.W //= scale_down
        w.H //= scale_down
        w.ndots = max(1, w.ndots // (scale_down * scale_down))
    return w


def truth(wl: Workload, x: np.ndarray, y: np.ndarray):
    return wl.field(np.asarray(x, np.float64), np.asarray(y, np.float64))
