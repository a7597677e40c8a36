"""One frame split across ranks by node-row bands (the parfor of
LocalICGN.m:91 and Subpb1.m:119 spread over GPUs instead of MATLAB workers).

The uniform node grid of MeshSetUp.m is cut into contiguous bands of node
rows, one per rank (nodes are x-fastest, so a band is a contiguous node
range).  Each rank holds only its band of the images -- the pixel rows its
search regions and subsets can reach, plus a margin -- and runs the
per-subset work (integer search, LocalICGN, Subpb1) on its own nodes.  The
per-subset results are all-gathered once per stage (one exchange per ADMM
iteration); the grid-wide steps that couple every node (Init's inpainting,
the bad-subset flags and refill, the beta sweep, Subproblem 2, nodal strain,
the dual update) are small and run replicated on every rank, so every rank
ends the frame with the whole field.

The frame follows main_ALDIC.m Sections 3-6 (FE Subproblem 2, no smoothing)
step for step; with exact integer search sums and per-subset IC-GN, a split
frame equals the single-process frame up to the rounding of band-local
coordinates (about 1e-12 px).

The arithmetic is delegated to a backend with the methods below, so the same
driver runs on the GPUs (DeviceBackend: this package's C ABI, one context per
rank) and, in the tests, on the CPU restatement.

    roi_sums(block)                    -> (sum, sum of squares, count), exact
    load(f, g, stats)                  band images (raw) + summed ROI sums
    search(gridx, gridy, w, step, s)   -> x, y, u, v (ny x nx) on the band grid
    icgn(coords, U0, w, tol)           -> U, F, iters, H21 (n x 21)
    subpb1(coords, UOld, FOld, vdual, H21, w, mu, tol) -> U, iters
    inpaint(M, N, z)                   Init's inpaint_nans(., 4)
    localicgn_post(M, N, iters, U, F)  -> U, F, bad count
    subpb1_post(M, N, iters, U)        -> U
    subpb2(M, N, h, beta, mu, U, F, udual, vdual) -> Uhat
    nodal_strain(M, N, h, U)           -> F
"""
from __future__ import annotations

import math

import numpy as np


# ------------------------------------------------------------------ geometry
def search_grid(W, H, gridx, gridy, winsize, step, search):
    """funIntegerSearch.m:14-25,90-91: (nx, ny, first template column, first
    template row), 1-based, after the ROI trimming."""
    sx, sy = (search, search) if np.ndim(search) == 0 else search
    gx1, gx2 = int(gridx[0]), int(gridx[1])
    gy1, gy2 = int(gridy[0]), int(gridy[1])
    hw, w15 = 0.5 * winsize, 1.5 * winsize
    while gx1 - sx - hw < 1:
        gx1 += 1
    while gy1 - sy - hw < 1:
        gy1 += 1
    while gx2 + w15 + sx > W:
        gx2 -= 1
    while gy2 + w15 + sy > H:
        gy2 -= 1
    nx = (gx2 - step - gx1) // step + 1 if gx2 - step >= gx1 else 0
    ny = (gy2 - step - gy1) // step + 1 if gy2 - step >= gy1 else 0
    return nx, ny, gx1, gy1


def node_bands(ny, world):
    """Contiguous node-row ranges [j0, j1), as even as possible."""
    base, extra = divmod(ny, world)
    out, j = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((j, j + k))
        j += k
    return out


def band_rows(H, gy1, step, winsize, search, j0, j1, margin=8):
    """0-based image rows [r0, r1) a band of node rows j0..j1-1 needs: its
    search regions (template rows ii-s .. ii+w+s, ii = gy1 + j step), the
    row reach of the search-grid trimming (ii + step + 1.5 w + s, so that the
    band grid keeps exactly these rows), and a margin for the IC-GN's
    displacement beyond the search radius and the bicubic stencil."""
    sy = search if np.ndim(search) == 0 else search[1]
    top = gy1 + j0 * step - sy - margin - 2                      # 1-based
    bot = gy1 + (j1 - 1) * step + step + int(math.ceil(1.5 * winsize)) + sy + margin + 2
    return max(0, top - 1), min(H, bot)


# ------------------------------------------------------------------ exchange
class Exchange:
    """All-gather of per-band row blocks over a torch.distributed group
    (NCCL on GPUs, gloo on CPUs).  Each rank passes its block (rows x cols,
    float64); the result is the blocks of all ranks in rank order."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.world = dist.get_world_size(group)
        self.device = device or torch.device("cpu")
        self.calls = 0

    def rows(self, block, counts):
        torch = self.torch
        block = np.ascontiguousarray(block, np.float64)
        width = block.shape[1] if block.ndim == 2 else 1
        pad = np.zeros((max(counts), width))
        pad[:len(block)] = block.reshape(len(block), width)
        t = torch.from_numpy(pad).to(self.device)
        outs = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(outs, t, group=self.group)
        self.calls += 1
        return np.concatenate([o.cpu().numpy()[:c] for o, c in zip(outs, counts)], 0)

    def sum3(self, a, b, c):
        torch = self.torch
        # integer sums below 2^53 stay exact in FP64
        t = torch.tensor([float(a), float(b), float(c)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        self.calls += 1
        return [int(v) for v in t.cpu().tolist()]


# ------------------------------------------------------------------ the frame
def select_beta(betas, e1, e2):
    """main_ALDIC.m:293-301: normalised error sum, its minimum, and the
    vertex of the parabola through the minimum and its neighbours in
    log10(beta)."""
    e1, e2 = np.asarray(e1), np.asarray(e2)
    es = (e1 - e1.mean()) / e1.std(ddof=1) + (e2 - e2.mean()) / e2.std(ddof=1)
    k = int(np.argmin(es))
    if 1 <= k <= len(betas) - 2:
        x = np.log10(betas[k - 1:k + 2])
        y = es[k - 1:k + 2]
        d01 = (y[1] - y[0]) / (x[1] - x[0])
        d12 = (y[2] - y[1]) / (x[2] - x[1])
        p1 = (d12 - d01) / (x[2] - x[0])
        p2 = d01 - p1 * (x[0] + x[1])
        return 10.0 ** (-p2 / 2.0 / p1)
    return float(betas[k])


def split_frame(backend, ex: Exchange, rank, f_raw, g_raw, winsize, step, search, gridx=None,
                gridy=None, tol=1e-2, mu=1e-3, n_admm=3, margin=8):
    """One frame of main_ALDIC.m Sections 3-6 with the per-subset work on
    this rank's node band.  f_raw, g_raw: the images (H, W) as the caller
    holds them; the backend receives only the band's rows.  Returns the
    whole-field result (identical on every rank)."""
    H, W = f_raw.shape
    gx = tuple(gridx) if gridx is not None else (1, W)
    gy = tuple(gridy) if gridy is not None else (1, H)
    nx, ny, gx1, gy1 = search_grid(W, H, gx, gy, winsize, step, search)
    bands = node_bands(ny, ex.world)
    j0, j1 = bands[rank]
    counts_nodes = [(b - a) * nx for a, b in bands]
    r0, r1 = band_rows(H, gy1, step, winsize, search, j0, j1, margin)
    # ROI rows (1-based, inclusive) this rank counts for the statistics of
    # funNormalizeImg.m: from its first node row's template row to the next
    # band's (the first and last ranks also take the ROI rows above and
    # below the grid), so every ROI row is counted once; the band holds them
    lo = gy[0] if rank == 0 else gy1 + j0 * step
    hi = gy[1] if rank == ex.world - 1 else gy1 + j1 * step - 1
    lo, hi = max(lo, gy[0]), min(hi, gy[1])
    if rank == 0:
        r0 = min(r0, gy[0] - 1)
    if rank == ex.world - 1:
        r1 = max(r1, gy[1])
    fb, gb = f_raw[r0:r1], g_raw[r0:r1]                           # the band this rank holds
    stats = []
    for img in (fb, gb):
        sl = img[lo - 1 - r0:hi - r0, gx[0] - 1:gx[1]] if hi >= lo else img[:0, :0]
        stats.append(ex.sum3(*backend.roi_sums(sl)))
    backend.load(fb, gb, stats)
    # Section 3: the band's search grid (its rows of the whole grid), Init
    gyb = (gy1 + j0 * step - r0, gy1 + j1 * step - r0)
    xb, yb, ub, vb = backend.search((gx1, gx[1]), gyb, winsize, step, search)
    blk = np.stack([np.asarray(a, np.float64).reshape(-1) for a in (xb, yb, ub, vb)], 1)
    blk[:, 1] += r0                                               # band -> image rows
    allg = ex.rows(blk, counts_nodes)
    x0, y0, u, v = (np.ascontiguousarray(allg[:, k]) for k in range(4))
    M, N, n = nx, ny, nx * ny
    U0 = np.empty(2 * n)
    U0[0::2] = backend.inpaint(M, N, u)
    U0[1::2] = backend.inpaint(M, N, v)
    k0, k1 = j0 * nx, j1 * nx
    coords_b = np.stack([x0[k0:k1], y0[k0:k1] - r0], 1)
    # Section 4: LocalICGN on the band, flags and refill on the whole grid
    Ub, Fb, itb, Hb = backend.icgn(coords_b, U0[2 * k0:2 * k1], winsize, tol)
    blk = np.concatenate([np.asarray(Ub).reshape(-1, 2), np.asarray(Fb).reshape(-1, 4),
                          np.asarray(itb, np.float64).reshape(-1, 1),
                          np.asarray(Hb).reshape(-1, 21)], 1)
    allg = ex.rows(blk, counts_nodes)
    U1 = np.ascontiguousarray(allg[:, 0:2]).reshape(-1)
    F1 = np.ascontiguousarray(allg[:, 2:6]).reshape(-1)
    it1 = allg[:, 6].astype(np.int32)
    H21 = np.ascontiguousarray(allg[:, 7:28])                     # n x 21
    U1, F1, nbad = backend.localicgn_post(M, N, it1, U1, F1)
    # Section 5: beta sweep and Subproblem 2, replicated
    ud, vd = np.zeros(4 * n), np.zeros(2 * n)
    betas = np.array([1e-3, math.sqrt(1e-5), 1e-2, math.sqrt(1e-3), 1e-1, math.sqrt(1e-1)]) * step * step * mu
    e1, e2 = [], []
    for b in betas:
        U2 = backend.subpb2(M, N, step, b, mu, U1, F1, ud, vd)
        F2 = backend.nodal_strain(M, N, step, U2)
        e1.append(np.linalg.norm(U1 - U2))
        e2.append(np.linalg.norm(F1 - F2))
    beta = select_beta(betas, e1, e2)
    U2 = backend.subpb2(M, N, step, beta, mu, U1, F1, ud, vd)
    F2 = backend.nodal_strain(M, N, step, U2)
    ud, vd = F2 - F1, U2 - U1
    # Section 6: ADMM, one all-gather of the band's Subpb1 results per step
    upd = []
    for _ in range(n_admm):
        U2old = U2.copy()
        Ub, itb = backend.subpb1(coords_b, U2[2 * k0:2 * k1], F2[4 * k0:4 * k1], vd[2 * k0:2 * k1],
                                 H21[k0:k1], winsize, mu, tol)
        blk = np.concatenate([np.asarray(Ub).reshape(-1, 2),
                              np.asarray(itb, np.float64).reshape(-1, 1)], 1)
        allg = ex.rows(blk, counts_nodes)
        U1 = backend.subpb1_post(M, N, allg[:, 2].astype(np.int32),
                                 np.ascontiguousarray(allg[:, 0:2]).reshape(-1))
        F1 = F2.copy()
        U2 = backend.subpb2(M, N, step, beta, mu, U1, F1, ud, vd)
        F2 = backend.nodal_strain(M, N, step, U2)
        upd.append(float(np.linalg.norm(U2old - U2) / math.sqrt(2 * n)))
        ud, vd = F2 - F1, U2 - U1
    return dict(M=M, N=N, x0=x0, y0=y0, U=U2, F=F2, beta=beta, bad_icgn=nbad, update_y=upd,
                band=(j0, j1), rows=(r0, r1), iters_icgn=it1)


class DeviceBackend:
    """The split frame's per-rank arithmetic on this rank's GPU through the C
    ABI: band images resident in the rank's own context, the global ROI
    statistics applied with aldic_set_stats, every call on the device."""

    def __init__(self, device=0, precision=None):
        import importlib
        self.A = importlib.import_module(__package__)
        self.api = self.A.api
        self.ctx = self.A.Context(device)
        self.precision = self.A.FP32 if precision is None else precision

    def roi_sums(self, block):
        b = np.asarray(block)
        if b.dtype.kind not in "ui":
            raise TypeError("the split frame takes 8- or 16-bit images")
        b = b.astype(np.int64)
        return int(b.sum()), int((b * b).sum()), int(b.size)

    def load(self, f, g, stats):
        st = []
        for s1, s2, n in stats:            # funNormalizeImg's mean and sample std
            m = s1 / n
            st += [m, math.sqrt((float(s2) - m * float(s1)) / (n - 1))]
        self.ctx.set_ref(np.ascontiguousarray(f))
        self.ctx.set_def(np.ascontiguousarray(g))
        self.A._lib.call("aldic_set_stats", self.ctx.h, self.api._ptr(np.asarray(st, np.float64)))
        self.shape = f.shape

    def search(self, gridx, gridy, w, step, search):
        import ctypes as C
        H, W = self.shape
        s = [int(search), int(search)] if np.ndim(search) == 0 else [int(search[0]), int(search[1])]
        gxa = (C.c_int * 2)(*gridx)
        gya = (C.c_int * 2)(*gridy)
        sa = (C.c_int * 2)(*s)
        nx, ny = C.c_int(), C.c_int()
        self.A._lib.call("aldic_search_dims", W, H, gxa, gya, int(w), int(step), sa, C.byref(nx),
                         C.byref(ny))
        outs = [np.empty((nx.value, ny.value)) for _ in range(5)]   # ny x nx column-major
        self.A._lib.call("aldic_int_search", self.ctx.h, gxa, gya, int(w), int(step), sa,
                         *[self.api._ptr(o) for o in outs], None)
        return tuple(o.T for o in outs[:4])

    def icgn(self, coords, U0, w, tol):
        return self.A.local_icgn(self.ctx, coords, U0, w, tol, self.precision)

    def subpb1(self, coords, UOld, FOld, vdual, H21, w, mu, tol):
        n = len(coords)
        U = np.empty(2 * n)
        it = np.empty(n, np.int32)
        cf = np.ascontiguousarray(np.asarray(coords, np.float64).T)
        Hc = np.ascontiguousarray(np.asarray(H21, np.float64).T)   # n x 21 column-major
        p = self.api._ptr
        self.A._lib.call("aldic_subpb1", self.ctx.h, p(cf), n, p(np.ascontiguousarray(UOld)),
                         p(np.ascontiguousarray(FOld)), p(np.ascontiguousarray(vdual)), p(Hc), None,
                         int(w), float(mu), float(tol), int(self.precision), p(U), p(it))
        return U, it

    def inpaint(self, M, N, z):
        return self.A.inpaint_nans(np.asarray(z, np.float64).reshape(N, M), 4).reshape(-1)

    def localicgn_post(self, M, N, iters, U, F):
        import ctypes as C
        U, F = np.array(U, np.float64), np.array(F, np.float64)
        nb = C.c_int()
        p = self.api._ptr
        self.A._lib.call("aldic_localicgn_post", self.ctx.h, M, N,
                         p(np.ascontiguousarray(iters, np.int32)), p(U), p(F), C.byref(nb))
        return U, F, nb.value

    def subpb1_post(self, M, N, iters, U):
        import ctypes as C
        U = np.array(U, np.float64)
        nb = C.c_int()
        p = self.api._ptr
        self.A._lib.call("aldic_subpb1_post", self.ctx.h, M, N,
                         p(np.ascontiguousarray(iters, np.int32)), p(U), C.byref(nb))
        return U

    def subpb2(self, M, N, h, beta, mu, U, F, ud, vd):
        out = np.empty(2 * M * N)
        p = self.api._ptr
        self.A._lib.call("aldic_subpb2", self.ctx.h, M, N, float(h), float(beta), float(mu),
                         p(np.ascontiguousarray(U)), p(np.ascontiguousarray(F)),
                         p(np.ascontiguousarray(ud)), p(np.ascontiguousarray(vd)), p(out))
        return out

    def nodal_strain(self, M, N, h, U):
        out = np.empty(4 * M * N)
        self.A._lib.call("aldic_nodal_strain", self.ctx.h, M, N, float(h),
                         self.api._ptr(np.ascontiguousarray(U)), self.api._ptr(out))
        return out

    def close(self):
        self.ctx.close()
