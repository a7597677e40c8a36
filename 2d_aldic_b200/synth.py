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
    hole: tuple | None = None      # (cx, cy, radius) of a circular hole
    min_size: int = 2              # quadtree elementMinSize (elements refined to 2x this)

    def mask(self):
        """ImgRefMask (H, W): 1 on the specimen, 0 in the hole."""
        if self.hole is None:
            return np.ones((self.H, self.W))
        return disk_mask(self.W, self.H, *self.hole)

    def images(self):
        f = speckle(self.W, self.H, self.ndots, self.seed, dtype=self.dtype,
                    scale=self.scale)
        g = warp(f, self.field, self.noise * self.scale, self.seed)
        return f, g

    def images_t(self, device="cpu"):
        """images() generated with torch (on the GPU when one is given): the
        same speckle draws and warp recipe, noise from torch's generator;
        fields must accept torch tensors."""
        import torch
        f = quantise_t(speckle_t(self.W, self.H, self.ndots, self.seed, device=device,
                                 scale=self.scale), self.dtype)
        ys, xs = torch.meshgrid(torch.arange(1, self.H + 1, dtype=torch.float64, device=device),
                                torch.arange(1, self.W + 1, dtype=torch.float64, device=device),
                                indexing="ij")
        X, Y = invert_t(self.field, xs, ys)
        g = bicubic_sample_t(f.to(torch.float64), X, Y)
        gen = torch.Generator(device=device).manual_seed(self.seed + 1000)
        g = g + self.noise * self.scale * torch.randn(g.shape, generator=gen, dtype=torch.float64,
                                                      device=device)
        return f, quantise_t(g, self.dtype)


def _affine_small(X, Y):
    return 0.5 + 0.01 * X, -0.3 + 0.005 * Y


def _xp(X):
    return np if isinstance(X, np.ndarray) else __import__("torch")


def _sine(X, Y):
    xp = _xp(X)
    return 2.0 * xp.sin(2 * np.pi * Y / 256.0), 1.5 * xp.cos(2 * np.pi * X / 256.0)


def _smooth_large(X, Y):
    xp = _xp(X)
    return 6.0 + 5.0 * xp.sin(2 * np.pi * Y / 2048.0), -4.0 + 5.0 * xp.cos(2 * np.pi * X / 2048.0)


def _large_shift(X, Y):
    """Displacements larger than a subset: 34-46 px in x, -24..-36 px in y,
    gradients up to 0.018 (numpy or torch arrays)."""
    xp = np if isinstance(X, np.ndarray) else __import__("torch")
    return (40.0 + 6.0 * xp.sin(2 * np.pi * Y / 2048.0),
            -30.0 + 6.0 * xp.cos(2 * np.pi * X / 2048.0))


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


def disk_mask(W, H, cx, cy, rad):
    """ImgRefMask of a plate with a circular hole: 0 inside the disk."""
    yy, xx = np.mgrid[1:H + 1, 1:W + 1]
    return ((xx - cx) ** 2 + (yy - cy) ** 2 >= rad * rad).astype(np.float64)


WORKLOADS = {
    # plain ALDIC, 512^2, 8000 dots, subset 20 / step 10, search +-20, FP64
    "plain512": Workload("plain512", 512, 512, 8000, 0, 20, 10, 20, 2.0, _affine_small,
                         tol=1e-3, fp64=True),
    # large uniform batch, 2048^2, 130k dots, subset 32 / step 8, sinusoidal
    "uniform2048": Workload("uniform2048", 2048, 2048, 130_000, 1, 32, 8, 16, 2.0, _sine),
    # learned-initial-guess evaluation frame: 4096^2, displacements up to
    # +-11 px with gradients up to 0.015 (inside the training distribution),
    # subset 32, step 16
    "learned4096": Workload("learned4096", 4096, 4096, 520_000, 5, 32, 16, 16, 2.0, _smooth_large),
    # plate with a hole of radius 300 px at the centre, quadtree mesh from a
    # 16 px grid, subset 32
    "plate2048": Workload("plate2048", 2048, 2048, 130_000, 2, 32, 16, 16, 2.0,
                          plate_hole(1024.0, 1024.0, 300.0), hole=(1024.0, 1024.0, 300.0)),
    # the same plate with the element range of its specification: a 64 px
    # grid (subset 64) refined toward the hole edge down to 8 px elements
    # (elementMinSize 4), element-sized subsets of 16-64 px
    "plate2048e": Workload("plate2048e", 2048, 2048, 130_000, 2, 64, 64, 16, 2.0,
                           plate_hole(1024.0, 1024.0, 300.0), hole=(1024.0, 1024.0, 300.0),
                           min_size=4),
    # displacements larger than the subset (up to 46 px): the multigrid
    # search (funIntegerSearchMg) initialises the frame; subset 32, step 16;
    # search 48 is the whole-field search radius that would cover the field
    "largeshift4096": Workload("largeshift4096", 4096, 4096, 520_000, 6, 32, 16, 48, 2.0,
                               _large_shift),
}


# ------------------------------------------------------ sequences (torch)
# The 16-bit sequence is generated with torch (on the GPU when one is given)
# from the same recipe: 50 frames of 4096^2 take seconds there instead of
# minutes in numpy.

def speckle_t(W: int, H: int, ndots: int, seed: int, device="cpu", bg: float = 20.0,
              amp=(80.0, 200.0), radius=(2.0, 4.0), scale: float = 1.0):
    """speckle() with the same draws, accumulated with torch; float64 (H, W)
    before quantisation."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    cx = rng.uniform(0, W, ndots)
    cy = rng.uniform(0, H, ndots)
    r = rng.uniform(radius[0], radius[1], ndots)
    A = rng.uniform(amp[0], amp[1], ndots)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)
    cx, cy, r, A = t(cx), t(cy), t(r), t(A)
    img = torch.zeros(H * W, dtype=torch.float64, device=device)
    R = 12
    off = torch.arange(-R, R + 1, device=device, dtype=torch.float64)
    chunk = 8192
    for s0 in range(0, ndots, chunk):
        e = min(ndots, s0 + chunk)
        px = torch.floor(cx[s0:e])[:, None, None] + off[None, None, :]
        py = torch.floor(cy[s0:e])[:, None, None] + off[None, :, None]
        d2 = (px - cx[s0:e, None, None]) ** 2 + (py - cy[s0:e, None, None]) ** 2
        val = A[s0:e, None, None] * torch.exp(-d2 / (r[s0:e, None, None] ** 2))
        ok = (px >= 0) & (px < W) & (py >= 0) & (py < H)
        idx = (py * W + px).expand_as(val)[ok].long()
        img.index_add_(0, idx, val[ok])
    return (img.reshape(H, W) + bg) * scale


def quantise_t(img, dtype):
    import torch
    info = np.iinfo(dtype)
    tdt = {np.uint8: torch.uint8, np.uint16: torch.uint16}[dtype]
    return torch.clamp(torch.round(img), info.min, info.max).to(torch.int32).to(tdt)


def bicubic_sample_t(img, x, y):
    """bicubic_sample() in torch (float64, 1-based coordinates)."""
    import torch
    H, W = img.shape
    im = img.to(torch.float64).reshape(-1)
    xf, yf = torch.floor(x), torch.floor(y)
    wx = keys_weights(x - xf)
    wy = keys_weights(y - yf)
    xi = xf.long() - 1
    yi = yf.long() - 1
    out = torch.zeros_like(x)
    for a in range(4):
        rows = torch.clamp(yi - 1 + a, 0, H - 1) * W
        acc = torch.zeros_like(x)
        for b in range(4):
            acc += wx[b] * im[rows + torch.clamp(xi - 1 + b, 0, W - 1)]
        out += wy[a] * acc
    return out


def invert_t(field, x, y, tol=1e-10, maxit=200):
    """X with X + u(X) = x (fixed-point iteration)."""
    X, Y = x.clone(), y.clone()
    for _ in range(maxit):
        u, v = field(X, Y)
        Xn, Yn = x - u, y - v
        err = max(float((Xn - X).abs().max()), float((Yn - Y).abs().max()))
        X, Y = Xn, Yn
        if err < tol:
            break
    return X, Y


@dataclasses.dataclass
class SequenceWorkload:
    """An image sequence: frame 0 is the speckle image, frame k (k >= 1) is it
    under the field k below plus noise (seed + 1000 + k).

    Field k (pixels, 1-based image coordinates, centre c):
      u = k*exx*(X - cx) + amp*sin(2*pi*(Y + drift*k)/period)
      v = k*eyy*(Y - cy) + amp*cos(2*pi*(X + drift*k)/period)
    i.e. a uniaxial stretch of eyy per frame with lateral contraction exx,
    plus a travelling sinusoid of amplitude amp."""
    name: str
    W: int
    H: int
    ndots: int
    seed: int
    n_frames: int
    winsize: int
    step: int
    search: int
    noise: float
    inc_unit: int | None
    exx: float = -0.0006
    eyy: float = 0.002
    amp: float = 0.5
    period: float = 512.0
    drift: float = 8.0
    scale: float = 257.0
    dtype: type = np.uint16
    tol: float = 1e-2
    n_admm: int = 3

    def field(self, k: int) -> Field:
        cx, cy = (self.W + 1) / 2.0, (self.H + 1) / 2.0

        def f(X, Y):
            xp = np if isinstance(X, np.ndarray) else __import__("torch")
            if k == 0:
                return 0.0 * X, 0.0 * Y
            u = k * self.exx * (X - cx) + self.amp * xp.sin(2 * math.pi * (Y + self.drift * k) / self.period)
            v = k * self.eyy * (Y - cy) + self.amp * xp.cos(2 * math.pi * (X + self.drift * k) / self.period)
            return u, v
        return f

    def frames(self, device="cpu"):
        """All frames as torch tensors of the integer type on device."""
        import torch
        f = speckle_t(self.W, self.H, self.ndots, self.seed, device=device, scale=self.scale)
        out = [quantise_t(f, self.dtype)]
        ys, xs = torch.meshgrid(torch.arange(1, self.H + 1, dtype=torch.float64, device=device),
                                torch.arange(1, self.W + 1, dtype=torch.float64, device=device),
                                indexing="ij")
        fq = out[0].to(torch.float64)
        for k in range(1, self.n_frames):
            X, Y = invert_t(self.field(k), xs, ys)
            g = bicubic_sample_t(fq, X, Y)
            gen = torch.Generator(device=device).manual_seed(self.seed + 1000 + k)
            g = g + self.noise * torch.randn(g.shape, generator=gen, dtype=torch.float64, device=device)
            out.append(quantise_t(g, self.dtype))
        return out

    def truth(self, k: int, r: int, x, y):
        """Displacement from frame r to frame k of the material points at
        (x, y) in frame r (the incremental reference's coordinates)."""
        import torch
        x = torch.as_tensor(np.asarray(x, np.float64))
        y = torch.as_tensor(np.asarray(y, np.float64))
        X, Y = invert_t(self.field(r), x, y) if r > 0 else (x, y)
        uk, vk = self.field(k)(X, Y)
        return (X + uk - x).numpy(), (Y + vk - y).numpy()


SEQUENCES = {
    # 50 frames of 4096^2 uint16 (intensities x257), 0.2 %/frame stretch in y
    # with 0.06 % lateral contraction, 0.5 px sinusoid, noise 30 grey levels;
    # subset 32, step 16; reference updated every 10 frames
    "sequence4096": SequenceWorkload("sequence4096", 4096, 4096, 520_000, 4, 50, 32, 16, 24, 30.0, 10),
}


def sequence(name: str, scale_down: int = 1, n_frames: int | None = None) -> SequenceWorkload:
    w = dataclasses.replace(SEQUENCES[name])
    if scale_down > 1:
        w.W //= scale_down
        w.H //= scale_down
        w.ndots = max(1, w.ndots // (scale_down * scale_down))
    if n_frames:
        w.n_frames = n_frames
    return w


def workload(name: str, scale_down: int = 1) -> Workload:
    """A named workload; scale_down > 1 shrinks the image (same density) for
    quick parity runs."""
    w = dataclasses.replace(WORKLOADS[name])
    if scale_down > 1:
        w.W //= scale_down
        w.H //= scale_down
        w.ndots = max(1, w.ndots // (scale_down * scale_down))
        if w.hole is not None:
            cx, cy, r = (v / scale_down for v in w.hole)
            w.hole = (cx, cy, r)
            w.field = plate_hole(cx, cy, r)
    return w


def truth(wl: Workload, x: np.ndarray, y: np.ndarray):
    return wl.field(np.asarray(x, np.float64), np.asarray(y, np.float64))
