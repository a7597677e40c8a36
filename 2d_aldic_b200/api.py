"""Reference-named host API over the C ABI (libaldic_b200.so).

Every function keeps the name, argument meaning and return values of the
reference MATLAB function it replaces (jyang526843/2D_ALDIC, cited per
function), so code written against the reference's frame loop can call these
one for one.  Layout conventions follow the reference after ReadImage's
transpose: an image Img(x, y) of W x H is a numpy array of shape (H, W)
(x fastest); U is interleaved [u1 v1 u2 v2 ...]; F is [F11 F21 F12 F22] per
node; coordinatesFEM is n x 2; HtempPar / HPar is n x 21.

Arrays may be numpy (host) arrays or CUDA torch tensors; outputs follow the
inputs (CUDA inputs give CUDA outputs, computed without host round trips).
All arithmetic runs in the sm_100a kernels -- there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time
from typing import Any

import numpy as np

from . import _lib
from ._lib import AldicError, FrameParams, FrameStats, QtFrameParams, QtFrameStats, call

try:  # torch is optional for host callers
    import torch
except Exception:  # pragma: no cover
    torch = None

U8, U16, F32, F64 = 0, 1, 2, 3
FP32, FP64 = 0, 1
# initial guess of a frame (ALDIC_INIT_* of the C ABI)
INIT_SEARCH, INIT_PREV, INIT_ZERO, INIT_EXTRAP, INIT_GIVEN, INIT_SEARCH_MG, INIT_GATED = 0, 1, 2, 3, 4, 5, 6
_DT = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.float32): F32,
       np.dtype(np.float64): F64}


# ------------------------------------------------------------------ arrays
def _is_cuda(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _ptr(a):
    if a is None:
        return None
    if _is_cuda(a):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


def _prep(a, dtype=np.float64):
    """numpy -> contiguous array of dtype; CUDA tensor -> contiguous tensor."""
    if a is None:
        return None
    if _is_cuda(a):
        tdt = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32,
               np.uint8: torch.uint8, np.uint16: torch.uint16}[np.dtype(dtype).type]
        return a.to(tdt).contiguous()
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _empty(like, shape, dtype=np.float64):
    if like is not None and _is_cuda(like):
        tdt = {np.float64: torch.float64, np.float32: torch.float32,
               np.int32: torch.int32}[np.dtype(dtype).type]
        return torch.empty(shape, dtype=tdt, device=like.device)
    return np.empty(shape, dtype=dtype)


def _first_cuda(*arrs):
    for a in arrs:
        if _is_cuda(a):
            return a
    return None


# ------------------------------------------------------------------ context
class Context:
    """A device context: images, gradients and work buffers resident on one
    GPU across calls (the MEX-session state of the reference's loop)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        call("aldic_ctx_create", int(device), C.byref(h))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aldic_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        """Use an existing CUDA stream (torch.cuda.Stream or raw handle)."""
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        call("aldic_ctx_set_stream", self.h, C.c_void_p(handle))

    # -- images
    def set_ref(self, img, roi=None, mask=None):
        H, W = img.shape
        dt = _dtype_code(img)
        r = (C.c_int * 4)(*roi) if roi is not None else None
        m = _prep(mask) if mask is not None else None
        call("aldic_set_ref", self.h, _ptr(_contig(img)), dt, W, H, r, _ptr(m))

    def set_def(self, img):
        call("aldic_set_def", self.h, _ptr(_contig(img)), _dtype_code(img))

    def set_fields(self, f=None, g=None, dfdx=None, dfdy=None, shape=None):
        ref = next(a for a in (f, g, dfdx, dfdy) if a is not None)
        H, W = ref.shape if shape is None else shape
        args = [_prep(a) for a in (f, g, dfdx, dfdy)]
        call("aldic_set_fields", self.h, *[_ptr(a) for a in args], W, H)

    def get_images(self, W, H, like=None):
        out = [_empty(like, (H, W)) for _ in range(4)]
        st = np.empty(4)
        call("aldic_get_images", self.h, *[_ptr(o) for o in out], _ptr(st))
        return (*out, st)


def _contig(a):
    if _is_cuda(a):
        return a.contiguous()
    return np.ascontiguousarray(a)


def _dtype_code(img) -> int:
    if _is_cuda(img):
        m = {torch.uint8: U8, torch.uint16: U16, torch.float32: F32, torch.float64: F64}
        return m[img.dtype]
    return _DT[np.asarray(img).dtype]


_ctx_lock = threading.Lock()
_ctxs: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    if device is None:
        device = torch.cuda.current_device() if torch is not None and torch.cuda.is_available() else 0
    with _ctx_lock:
        if device not in _ctxs:
            _ctxs[device] = Context(device)
        return _ctxs[device]


def _ctx_for(*arrs) -> Context:
    t = _first_cuda(*arrs)
    return default_context(t.device.index if t is not None else None)


# ------------------------------------------------------------------ a3
def ba_interp2(F, X, Y, method: str = "cubic"):
    """Z = ba_interp2(F, X, Y, [method]) -- ba_interp2.cpp:318-335.

    F is MATLAB's M x N (x P) column-major image: pass the numpy array of
    shape (N, M) or (P, N, M) (its transpose in C order).  X indexes columns
    (N) and Y rows (M), 1-based; the method string is ignored (cubic only, as
    in the reference).  All of F, X, Y must be float64 or all float32."""
    dt = (F.dtype if not _is_cuda(F) else {torch.float64: np.float64, torch.float32: np.float32}[F.dtype])
    dt = np.dtype(dt)
    if dt not in (np.dtype(np.float64), np.dtype(np.float32)):
        raise TypeError("ba_interp2 takes only double or single arguments for IMG,X,Y, and all "
                        "must have the same class")
    for a in (X, Y):
        adt = a.dtype if not _is_cuda(a) else {torch.float64: np.float64, torch.float32: np.float32}.get(a.dtype)
        if np.dtype(adt) != dt:
            raise TypeError("ba_interp2 takes only double or single arguments for IMG,X,Y, and "
                            "all must have the same class")
    if tuple(X.shape) != tuple(Y.shape):
        raise ValueError("X, Y should have the same size")
    Fc, Xc, Yc = _contig(F), _contig(X), _contig(Y)
    if Fc.ndim == 2:
        Pn, N, M = 1, Fc.shape[0], Fc.shape[1]
    else:
        Pn, N, M = Fc.shape
    n = int(np.prod(X.shape)) if not _is_cuda(X) else X.numel()
    out = _empty(_first_cuda(F, X, Y), (Pn,) + tuple(X.shape), dt.type)
    fn = "aldic_ba_interp2_f64" if dt == np.dtype(np.float64) else "aldic_ba_interp2_f32"
    stream = None
    if _first_cuda(F, X, Y) is not None:
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    call(fn, _ptr(Fc), M, N, Pn, _ptr(Xc), _ptr(Yc), n, _ptr(out), stream)
    return out[0] if Pn == 1 else out


# ------------------------------------------------------------------ a1/a2
def funNormalizeImg(Img, gridxyROIRange):
    """[ImgNormalized, gridxyROIRange] = funNormalizeImg(Img, gridxyROIRange)
    -- funNormalizeImg.m:1.  Img is a list of (H, W) images."""
    gx = list(gridxyROIRange["gridx"])
    gy = list(gridxyROIRange["gridy"])
    H, W = Img[0].shape
    gx = [max(gx[0], 1), min(gx[1], W)]
    gy = [max(gy[0], 1), min(gy[1], H)]
    ctx = _ctx_for(*Img)
    out = []
    for im in Img:
        o = _empty(_first_cuda(im), (H, W))
        call("aldic_normalize", ctx.h, _ptr(_contig(im)), _dtype_code(im), W, H,
             (C.c_int * 4)(gx[0], gx[1], gy[0], gy[1]), _ptr(o), None)
        out.append(o)
    return out, {"gridx": gx, "gridy": gy}


def funImgGradient(ImgRef, ImgDef=None, ImgRefMask=None):
    """Df = funImgGradient(ImgRef, ImgDef, [ImgRefMask]) -- funImgGradient.m:1.
    Returns a dict with DfDx, DfDy ((H-6) x (W-6), i.e. MATLAB's
    (W-6) x (H-6)), DfCropWidth = 3, DfAxis and imgSize = (W, H)."""
    H, W = ImgRef.shape
    f = _prep(ImgRef)
    m = _prep(ImgRefMask) if ImgRefMask is not None else None
    gx = _empty(_first_cuda(f), (H, W))
    gy = _empty(_first_cuda(f), (H, W))
    call("aldic_gradient", _ctx_for(f).h, _ptr(f), W, H, _ptr(m), _ptr(gx), _ptr(gy))
    return {"DfDx": gx[3:H - 3, 3:W - 3], "DfDy": gy[3:H - 3, 3:W - 3], "DfCropWidth": 3,
            "DfAxis": [4, W - 3, 4, H - 3], "imgSize": (W, H),
            "ImgRefMask": ImgRefMask if ImgRefMask is not None else None}


def _df_full(Df, shape, like):
    H, W = shape
    if _is_cuda(like):
        fx = torch.zeros((H, W), dtype=torch.float64, device=like.device)
        fy = torch.zeros_like(fx)
    else:
        fx = np.zeros((H, W))
        fy = np.zeros((H, W))
    fx[3:H - 3, 3:W - 3] = Df["DfDx"]
    fy[3:H - 3, 3:W - 3] = Df["DfDy"]
    return fx, fy


def _load_fields(ctx, ImgRef, ImgDef, Df):
    H, W = ImgRef.shape
    fx, fy = _df_full(Df, (H, W), ImgRef)
    ctx.set_fields(ImgRef, ImgDef, fx, fy)


# ------------------------------------------------------------------ a4/a5
def funIntegerSearch(f, g, tempSizeOfSearchRegion, gridx, gridy, winsize, winstepsize,
                     tempNoOfInitPt=0, *varargin, qfactors: bool = True, ctx: Context | None = None):
    """[x,y,u,v,cc] = funIntegerSearch(f,g,tempSizeOfSearchRegion,gridx,gridy,
    winsize,winstepsize,0,winstepsize) -- funIntegerSearch.m:3 (whole field).

    f, g: images (H, W); integer images (uint8/uint16) give exact correlation
    maps.  Returns x, y, u, v as ny x nx arrays and cc = {'max': ...,
    'qfactors': n x 2}."""
    if tempNoOfInitPt != 0:
        raise NotImplementedError("only the whole-field search (tempNoOfInitPt = 0) is on the "
                                  "GPU path; the seed-point mode is interactive in the reference")
    s = tempSizeOfSearchRegion
    s = [int(s), int(s)] if np.ndim(s) == 0 else [int(s[0]), int(s[1])]
    ctx = ctx or _ctx_for(f, g)
    H, W = f.shape
    if _dtype_code(f) in (U8, U16):
        # the reference searches images normalised over gridxyROIRange (main_ALDIC.m
        # Section 2): the ROI statistics set the value the correlation pads with
        ctx.set_ref(f, roi=(int(gridx[0]), int(gridx[-1]), int(gridy[0]), int(gridy[-1])))
        ctx.set_def(g)
    else:
        ctx.set_fields(_prep(f), _prep(g), _zeros_like_img(f), _zeros_like_img(f))
    gxa = (C.c_int * 2)(int(gridx[0]), int(gridx[-1]))
    gya = (C.c_int * 2)(int(gridy[0]), int(gridy[-1]))
    sa = (C.c_int * 2)(*s)
    nx, ny = C.c_int(), C.c_int()
    call("aldic_search_dims", W, H, gxa, gya, int(winsize), int(winstepsize), sa, C.byref(nx),
         C.byref(ny))
    nx, ny = nx.value, ny.value
    like = _first_cuda(f, g)
    outs = [_empty(like, (nx, ny)) for _ in range(5)]  # column-major ny x nx
    q = _empty(like, (2, nx * ny)) if qfactors else None
    call("aldic_int_search", ctx.h, gxa, gya, int(winsize), int(winstepsize), sa,
         *[_ptr(o) for o in outs], _ptr(q))
    x, y, u, v, cmax = (o.T for o in outs)
    cc = {"max": cmax, "qfactors": q.T if q is not None else None, "A": []}
    return x, y, u, v, cc


def funIntegerSearchMg(f, g, gridx, gridy, winsize, winstepsize, *varargin,
                       ctx: Context | None = None, info: dict | None = None):
    """[xGrid,yGrid,uGrid,vGrid,cc] = funIntegerSearchMg(f,g,gridx,gridy,
    winsize,winstepsize,winstepsize) -- funIntegerSearchMg.m:1, the multigrid
    search of IntegerSearch.m:117-120 for large displacements.

    f, g: images (H, W).  Returns x, y, u, v as ny x nx arrays on the node
    grid gridx(1):step:gridx(2) (its borders follow the displacements of the
    outermost regions) and cc = {'max': ny x nx, 'qfactors': (nx*ny) x 2 in
    column-major grid order, as cc.qfactors = [qf_1Grid(:), qf_2Grid(:)]}.
    info, when given, receives the level count, the last-level region count,
    the regions whose correlation raised and the level-1 (whole ROI) shift."""
    ctx = ctx or _ctx_for(f, g)
    H, W = f.shape
    if _dtype_code(f) in (U8, U16):
        # the reference searches images normalised over gridxyROIRange (main_ALDIC.m
        # Section 2): the ROI statistics set the value the correlation pads with
        ctx.set_ref(f, roi=(int(gridx[0]), int(gridx[-1]), int(gridy[0]), int(gridy[-1])))
        ctx.set_def(g)
    else:
        ctx.set_fields(_prep(f), _prep(g), _zeros_like_img(f), _zeros_like_img(f))
    gxa = (C.c_int * 2)(int(gridx[0]), int(gridx[-1]))
    gya = (C.c_int * 2)(int(gridy[0]), int(gridy[-1]))
    step = int(winstepsize if np.ndim(winstepsize) == 0 else winstepsize[0])
    cap = (W // step + 1) * (H // step + 1)
    like = _first_cuda(f, g)
    outs = [_empty(like, (cap,)) for _ in range(5)]
    q = _empty(like, (2, cap))
    nx, ny = C.c_int(), C.c_int()
    inf = np.zeros(10)
    call("aldic_int_search_mg", ctx.h, gxa, gya, int(winsize), step, C.byref(nx), C.byref(ny), cap,
         *[_ptr(o) for o in outs], _ptr(q), _ptr(inf))
    nx, ny = nx.value, ny.value
    n = nx * ny
    x, y, u, v, cmax = (o[:n].reshape(ny, nx) for o in outs)
    qs = q.reshape(-1)[:2 * n].reshape(2, ny, nx)
    if _is_cuda(qs):
        qf = torch.stack([qs[0].T.reshape(-1), qs[1].T.reshape(-1)], 1)
    else:
        qf = np.stack([qs[0].T.reshape(-1), qs[1].T.reshape(-1)], 1)
    if info is not None:
        info.update(levels=int(inf[0]), regions=int(inf[1]), failed=int(inf[2]),
                    level1_u=float(inf[3]), level1_v=float(inf[4]), level1_cc=float(inf[5]),
                    ms_level1=float(inf[6]), ms_levels=float(inf[7]), ms_last_level=float(inf[8]),
                    ms_gridfit=float(inf[9]))
    return x, y, u, v, {"max": cmax, "qfactors": qf, "A": []}


def _zeros_like_img(f):
    if _is_cuda(f):
        return torch.zeros(f.shape, dtype=torch.float64, device=f.device)
    return np.zeros(f.shape)


def IntegerSearch(ImgRef, ImgDef, file_name, DICpara):
    """[DICpara,x0,y0,u,v,cc] = IntegerSearch(ImgRef,ImgDef,file_name,DICpara)
    -- IntegerSearch.m:1, non-interactive.  DICpara['InitFFTSearchMethod']
    (default 1) picks the whole-field search, whose zone comes from
    DICpara['SizeOfFFTSearchRegion'] instead of input(), or -- for any value
    other than 1 and 2 -- the multigrid search funIntegerSearchMg
    (IntegerSearch.m:117-120).  The seed-point method 2 is interactive in the
    reference (ginput) and is not available."""
    method = DICpara.get("InitFFTSearchMethod", 1)
    roi = DICpara["gridxyROIRange"]
    if method == 2:
        raise NotImplementedError("InitFFTSearchMethod = 2 picks seed points with ginput")
    if method == 1:
        s = DICpara.get("SizeOfFFTSearchRegion")
        if s is None:
            raise ValueError("DICpara['SizeOfFFTSearchRegion'] is required (the reference asks "
                             "for it interactively)")
        x0, y0, u, v, cc = funIntegerSearch(ImgRef, ImgDef, s, roi["gridx"], roi["gridy"],
                                            DICpara["winsize"], DICpara["winstepsize"], 0,
                                            DICpara["winstepsize"])
    else:
        x0, y0, u, v, cc = funIntegerSearchMg(ImgRef, ImgDef, roi["gridx"], roi["gridy"],
                                              DICpara["winsize"], DICpara["winstepsize"],
                                              DICpara["winstepsize"])
    DICpara = dict(DICpara, InitFFTSearchMethod=method)
    mask = DICpara.get("ImgRefMask")
    if mask is not None:  # IntegerSearch.m:68-73, :125-131
        xi = np.asarray(x0, int).ravel() - 1
        yi = np.asarray(y0, int).ravel() - 1
        hole = np.asarray(mask)[yi, xi].reshape(np.shape(x0)).astype(float)
        hole[hole == 0] = np.nan
        u = u * hole
        v = v * hole
    return DICpara, x0, y0, u, v, cc


# ------------------------------------------------------------------ a6
def MeshSetUp(x, y, DICpara):
    """DICmesh = MeshSetUp(x, y, DICpara) -- MeshSetUp.m:23-39, 80-89."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    N, M = x.shape  # N vertical (y), M horizontal (x)
    xt, yt = x.T, y.T
    coords = np.stack([xt.ravel(order="F"), yt.ravel(order="F")], axis=1)
    j, i = np.meshgrid(np.arange(1, N), np.arange(1, M), indexing="ij")
    i, j = i.ravel(), j.ravel()
    elems = np.stack([(j - 1) * M + i, (j - 1) * M + i + 1, j * M + i + 1, j * M + i], axis=1)
    H = DICpara.get("ImgSize", (0, 0))[1]
    return {"coordinatesFEM": coords, "elementsFEM": elems.astype(np.int64), "dirichlet": [],
            "neumann": [], "x0": xt, "y0": yt, "M": M, "N": N,
            "y0World": H + 1 - yt,
            "coordinatesFEMWorld": np.stack([coords[:, 0], H + 1 - coords[:, 1]], axis=1)}


def Init(u, v, Phi, x, y, index=0):
    """U0 = Init(u, v, Phi, x, y, 0) -- Init.m:13,168-179: NaNs filled by the
    4-neighbour spring inpainting (inpaint_nans method 4, on the GPU), then
    interleaved x-fastest."""
    if index != 0:
        raise NotImplementedError("Init index 1 (outlier spring test) is not on the GPU path")
    u = np.array(u, np.float64)
    v = np.array(v, np.float64)
    ny, nx = u.shape
    z = np.stack([u.ravel(), v.ravel()])  # row-major (ny, nx) == x fastest
    call("aldic_inpaint_springs", default_context().h, nx, ny, 2, _ptr(z))
    U0 = np.empty(2 * nx * ny)
    U0[0::2] = z[0]
    U0[1::2] = z[1]
    return U0


# ------------------------------------------------------------------ a7/a8
def _winsize_arr(winsize, n, like):
    if np.ndim(winsize) == 0:
        return None, int(winsize)
    return _prep(np.asarray(winsize, np.int32) if not _is_cuda(winsize) else winsize, np.int32), 0


def local_icgn(ctx: Context, coords, U0, winsize, tol, precision=FP32):
    """Batch funICGN over every node on the images resident in ctx.  Returns
    U (2n), F (4n), ConvItPerEle (n), HtempPar (n x 21)."""
    cf = _coords_cm(coords)
    n = cf.shape[-1] if not _is_cuda(cf) else cf.shape[-1]
    like = _first_cuda(coords, U0)
    U0p = _prep(U0)
    wa, w = _winsize_arr(winsize, n, like)
    U = _empty(like, (2 * n,))
    F = _empty(like, (4 * n,))
    it = _empty(like, (n,), np.int32)
    Hp = _empty(like, (21, n))
    call("aldic_icgn", ctx.h, _ptr(cf), n, _ptr(U0p), _ptr(wa), w, float(tol), int(precision),
         _ptr(U), _ptr(F), _ptr(it), _ptr(Hp))
    return U, F, it, Hp.T


def _coords_cm(coords):
    """n x 2 coordinatesFEM -> column-major [x1..xn y1..yn] buffer of shape (2, n)."""
    if _is_cuda(coords):
        return coords.to(torch.float64).t().contiguous()
    return np.ascontiguousarray(np.asarray(coords, np.float64).reshape(-1, 2).T)


def funICGN(U0, x0, y0, Df, ImgRef, ImgDef, winsize, tol, ICGNmethod="GaussNewton"):
    """[U,F,stepwithinwhile,HGlobal] = funICGN(U0,x0,y0,Df,ImgRef,ImgDef,
    winsize,tol,ICGNmethod) -- funICGN.m:1 for one subset (FP64)."""
    _check_method(ICGNmethod)
    ctx = _ctx_for(ImgRef)
    _load_fields(ctx, ImgRef, ImgDef, Df)
    U, F, it, Hp = local_icgn(ctx, np.array([[x0, y0]], float), np.asarray(U0, float)[:2],
                              winsize, tol, FP64)
    return U, F, int(it[0]), np.asarray(Hp)[0]


def _check_method(m):
    if m not in ("GaussNewton", "Gauss-Newton", None):
        # the reference's LevenbergMarquardt branch calls ImgDef.eval on a
        # numeric array and always errors (funICGN.m:199)
        raise NotImplementedError("only ICGNmethod='GaussNewton' exists on the reference's "
                                  "working path")


def LocalICGN(U0, coordinatesFEM, Df, ImgRef, ImgDef, DICpara, ICGNmethod="GaussNewton",
              tol=1e-2, precision=FP64):
    """[U,F,HtempPar,LocalTime,ConvItPerEle,LocalICGNBadPtNum] = LocalICGN(U0,
    coordinatesFEM,Df,ImgRef,ImgDef,DICpara,ICGNmethod,tol) -- LocalICGN.m:1,
    including the bad-subset flags and refill of :117-161 (refill by spring
    inpainting on the node grid)."""
    _check_method(ICGNmethod)
    ctx = _ctx_for(ImgRef)
    t0 = time.perf_counter()
    _load_fields(ctx, ImgRef, ImgDef, Df)
    U, F, it, Hp = local_icgn(ctx, coordinatesFEM, U0, DICpara["winsize"], tol, precision)
    M, N = _grid_dims(coordinatesFEM)
    bad = C.c_int()
    call("aldic_localicgn_post", ctx.h, M, N, _ptr(_prep(it, np.int32)), _ptr(U), _ptr(F),
         C.byref(bad))
    return U, F, Hp, time.perf_counter() - t0, it, bad.value


def _grid_dims(coords):
    c = coords.cpu().numpy() if _is_cuda(coords) else np.asarray(coords)
    M = len(np.unique(c[:, 0]))
    N = len(np.unique(c[:, 1]))
    if M * N != c.shape[0]:
        raise ValueError("coordinatesFEM is not a uniform M x N grid")
    return M, N


# ------------------------------------------------------------------ a9
def funICGN_Subpb1(x0, y0, Df, ImgRef, ImgDef, winsize, H, beta, mu, udual, vdual, UOld, FOld,
                   tol, ICGNmethod="GaussNewton"):
    """[U,H,stepwithinwhile] = funICGN_Subpb1(...) -- funICGN_Subpb1.m:1 for
    one subset (FP64).  H is the 6x6 Hessian of the subset."""
    _check_method(ICGNmethod)
    ctx = _ctx_for(ImgRef)
    _load_fields(ctx, ImgRef, ImgDef, Df)
    Hm = np.asarray(H, float)
    H21 = np.array([Hm[r, c] for c in range(6) for r in range(c, 6)]).reshape(21, 1)
    U = np.empty(2)
    it = np.empty(1, np.int32)
    coords = np.array([[x0], [y0]], float)
    wa, w = _winsize_arr(winsize, 1, None)
    call("aldic_subpb1", ctx.h, _ptr(coords), 1, _ptr(np.asarray(UOld, float)[:2].copy()),
         _ptr(np.asarray(FOld, float)[:4].copy()), _ptr(np.asarray(vdual, float)[:2].copy()),
         _ptr(H21), _ptr(wa), w, float(mu), float(tol), FP64, _ptr(U), _ptr(it))
    return U, Hm, int(it[0])


def Subpb1(UOld, FOld, udual, vdual, coordinatesFEM, Df, ImgRef, ImgDef, mu, beta, HPar,
           ALSolveStep, DICpara, ICGNmethod="GaussNewton", tol=1e-2, precision=FP64):
    """[U,HPar,ALSub1Time,ConvItPerEle,LocalICGNBadPtNum] = Subpb1(...) --
    Subpb1.m:1 (ALSolveStep > 1) with the gridfit 'springs' post-processing
    of :186-199.  HPar: n x 21 array (or the reference's 21-cell of n)."""
    _check_method(ICGNmethod)
    if ALSolveStep <= 1:
        raise ValueError("Subpb1 is called with ALSolveStep > 1 in the reference's loop "
                         "(HPar is only read then)")
    ctx = _ctx_for(ImgRef)
    t0 = time.perf_counter()
    _load_fields(ctx, ImgRef, ImgDef, Df)
    Hp = np.column_stack(HPar) if isinstance(HPar, (list, tuple)) else HPar
    H21 = _prep(Hp.T if not _is_cuda(Hp) else Hp.t())
    cf = _coords_cm(coordinatesFEM)
    n = cf.shape[-1]
    like = _first_cuda(coordinatesFEM, UOld)
    U = _empty(like, (2 * n,))
    it = _empty(like, (n,), np.int32)
    wa, w = _winsize_arr(DICpara["winsize"], n, like)
    call("aldic_subpb1", ctx.h, _ptr(cf), n, _ptr(_prep(UOld)), _ptr(_prep(FOld)),
         _ptr(_prep(vdual)), _ptr(H21), _ptr(wa), w, float(mu), float(tol), int(precision),
         _ptr(U), _ptr(it))
    M, N = _grid_dims(coordinatesFEM)
    bad = C.c_int()
    call("aldic_subpb1_post", ctx.h, M, N, _ptr(it), _ptr(U), C.byref(bad))
    return U, HPar, time.perf_counter() - t0, it, bad.value


# ------------------------------------------------------------------ a10/a11
def Subpb2(DICmesh, beta, mu, U, F, udual, vdual, alpha=0, GaussPtOrder=2):
    """Uhat = Subpb2(DICmesh,beta,mu,U,F,udual,vdual,alpha,GaussPtOrder) --
    Subpb2.m:1 on the uniform mesh (dirichlet and neumann empty)."""
    if alpha != 0:
        raise NotImplementedError("alpha != 0 is never used by the reference's loop")
    if len(DICmesh.get("dirichlet", [])) or len(DICmesh.get("neumann", [])):
        raise NotImplementedError("Dirichlet/Neumann nodes belong to the quadtree path")
    coords = DICmesh["coordinatesFEM"]
    c = coords.cpu().numpy() if _is_cuda(coords) else np.asarray(coords)
    step = abs(c[0, 0] - c[1, 0])  # Subpb2.m:29
    M, N = int(DICmesh["M"]), int(DICmesh["N"])
    like = _first_cuda(U, F)
    out = _empty(like, (2 * M * N,))
    ctx = _ctx_for(U)
    call("aldic_subpb2", ctx.h, M, N, float(step), float(beta), float(mu), _ptr(_prep(U)),
         _ptr(_prep(F)), _ptr(_prep(udual)), _ptr(_prep(vdual)), _ptr(out))
    return out


def ComputeStrain(ULocal, FLocal, DICmesh, DICpara, ctx: Context | None = None):
    """ComputeStrain.m: strains on the uniform mesh.  DICpara keys
    MethodToComputeStrain (0 solved F, 1 central differences, 2 plane
    fitting, 3 finite elements; default 3), StrainType (0 infinitesimal,
    1 Eulerian, 2 Green-Lagrangian; default 0) and, for method 2, PlaneFitRad
    (the half window the reference asks for interactively).  Returns a dict
    with FStrain and FStrainFinite (4n, [F11 F21 F12 F22]) and FStrainWorld
    (the nodes inside the Rad ring, the F21 and F12 slots negated for the
    upward y axis).  Method 3 keeps funGlobal_NodalStrainAvg's slot order
    [du/dx du/dy dv/dx dv/dy], which ComputeStrain.m then reads as
    [F11 F21 F12 F22], as the reference does."""
    ctx = ctx or default_context()
    method = int(DICpara.get("MethodToComputeStrain", 3))
    stype = int(DICpara.get("StrainType", 0))
    rad = {0: 0, 1: 1, 2: int(DICpara.get("PlaneFitRad", 2)), 3: 1}[method]
    M, N = int(DICmesh["M"]), int(DICmesh["N"])
    h = float(np.mean(DICpara["winstepsize"]))
    U = np.ascontiguousarray(ULocal, np.float64) if ULocal is not None else None
    F = np.ascontiguousarray(FLocal, np.float64) if FLocal is not None else None
    fs = np.empty(4 * M * N)
    ff = np.empty(4 * M * N)
    call("aldic_compute_strain", ctx.h, M, N, h, method, rad, stype, _ptr(U), _ptr(F), _ptr(fs), _ptr(ff))
    i, j = np.meshgrid(np.arange(M), np.arange(N))
    k = (j * M + i)[rad:N - rad, rad:M - rad].reshape(-1)
    world = ff.reshape(-1, 4)[k].copy()
    world[:, 1:3] *= -1
    return {"FStrain": fs, "FStrainFinite": ff, "FStrainWorld": world.reshape(-1)}


def subpb2_fd(M, N, winstepsize, beta, mu, U, F, udual, vdual, ctx: Context | None = None):
    """The finite-difference Subproblem 2 of main_ALDIC.m:243-259 (interior
    nodes solve (beta D'D + mu I) x = beta D'(F - udual) + mu (U - vdual),
    D = funDerivativeOp of the interior grid; border nodes keep U)."""
    ctx = ctx or _ctx_for(U)
    Ua, Fa, ua, va = _prep(U), _prep(F), _prep(udual), _prep(vdual)
    out = _empty(_first_cuda(Ua), (2 * M * N,))
    call("aldic_subpb2_fd", ctx.h, int(M), int(N), float(winstepsize), float(beta), float(mu),
         _ptr(Ua), _ptr(Fa), _ptr(ua), _ptr(va), _ptr(out))
    return out


def fd_strain(M, N, winstepsize, U, ctx: Context | None = None):
    """F = funDerivativeOp(M, N, winstepsize) * U (main_ALDIC.m:259)."""
    ctx = ctx or _ctx_for(U)
    Ua = _prep(U)
    out = _empty(_first_cuda(Ua), (4 * M * N,))
    call("aldic_fd_strain", ctx.h, int(M), int(N), float(winstepsize), _ptr(Ua), _ptr(out))
    return out


def funGlobal_NodalStrainAvg(coordinatesFEM, elementsFEM, U, GaussPtOrder=2):
    """StrainNodalPt = funGlobal_NodalStrainAvg(coordinatesFEM,elementsFEM,U,
    GaussPtOrder) -- funGlobal_NodalStrainAvg.m:1 on the uniform mesh."""
    M, N = _grid_dims(coordinatesFEM)
    c = coordinatesFEM.cpu().numpy() if _is_cuda(coordinatesFEM) else np.asarray(coordinatesFEM)
    step = abs(c[1, 0] - c[0, 0])
    out = _empty(_first_cuda(U), (4 * M * N,))
    call("aldic_nodal_strain", _ctx_for(U).h, M, N, float(step), _ptr(_prep(U)), _ptr(out))
    return out


# ------------------------------------------------------------------ a14
def gridfit_springs(M, N, fields):
    """gridfit(x, y, z, xnodes, ynodes, 'regularizer', 'springs') for data on
    the nodes of an M x N grid (NaN = no data); fields: (nf, M*N)."""
    z = _prep(fields).reshape(-1, M * N) if not _is_cuda(fields) else _prep(fields).reshape(-1, M * N)
    out = _empty(_first_cuda(fields), tuple(z.shape))
    call("aldic_gridfit_springs", _ctx_for(fields).h, M, N, z.shape[0], _ptr(z), _ptr(out))
    return out


def inpaint_nans(A, method=4):
    """B = inpaint_nans(A, 4) -- spring method of inpaint_nans.m."""
    if method != 4:
        raise NotImplementedError("only the spring method (4) is used on the reference's path")
    A = np.array(A, np.float64)
    ny, nx = A.shape
    call("aldic_inpaint_springs", default_context().h, nx, ny, 1, _ptr(A))
    return A


def funSmoothDisp(ULocal, DICmesh, DICpara=None):
    """ULocal = funSmoothDisp(ULocal,DICmesh,DICpara) -- funSmoothDisp.m with
    the default filter (3x3, sigma 0.5), two passes."""
    M, N = int(DICmesh["M"]), int(DICmesh["N"])
    v = _prep(ULocal).copy() if not _is_cuda(ULocal) else _prep(ULocal).clone()
    call("aldic_smooth", _ctx_for(ULocal).h, M, N, 2, _ptr(v))
    return v


def funSmoothStrain(F, DICmesh, DICpara=None):
    """F = funSmoothStrain(F,DICmesh,DICpara) -- funSmoothStrain.m, default
    filter, two passes."""
    M, N = int(DICmesh["M"]), int(DICmesh["N"])
    v = _prep(F).copy() if not _is_cuda(F) else _prep(F).clone()
    call("aldic_smooth", _ctx_for(F).h, M, N, 4, _ptr(v))
    return v


# ------------------------------------------------------------------ a12
class ALDIC:
    """One-frame AL-DIC driver (main_ALDIC.m Sections 3-6) on a context.

        al = ALDIC(winsize=32, step=8, search=16)
        al.set_images(f, g)           # raw uint8/uint16/float images (H, W)
        res = al.frame()              # dict: x0, y0, U, F, iters, stats
    """

    def __init__(self, winsize, step, search, tol=1e-2, mu=1e-3, beta=0.0, n_admm=3,
                 precision=FP32, smooth=False, gridx=(0, 0), gridy=(0, 0), use_graph=True,
                 device=None, ctx: Context | None = None, subpb2: str = "fe"):
        self.ctx = ctx or default_context(device)
        p = FrameParams()
        p.winsize, p.step = int(winsize), int(step)
        s = (search, search) if np.ndim(search) == 0 else search
        p.search[0], p.search[1] = int(s[0]), int(s[1])
        p.gridx[0], p.gridx[1] = gridx
        p.gridy[0], p.gridy[1] = gridy
        p.tol, p.mu, p.beta, p.n_admm = float(tol), float(mu), float(beta), int(n_admm)
        p.tol2 = 0.0
        p.precision, p.smooth, p.use_graph = int(precision), int(bool(smooth)), int(bool(use_graph))
        if subpb2 not in ("fe", "fd"):
            raise ValueError("subpb2 must be 'fe' (Subpb2.m) or 'fd' (finite differences)")
        p.subpb2_fd = int(subpb2 == "fd")
        self.p = p
        self.node_grid = None   # grid of the last multigrid-search frame
        self.shape = None

    def set_images(self, f=None, g=None, roi=None, mask=None):
        if f is not None:
            self.ctx.set_ref(f, roi=roi, mask=mask)
            self.shape = tuple(f.shape)
        if g is not None:
            self.ctx.set_def(g)

    def dims(self):
        M, N = C.c_int(), C.c_int()
        call("aldic_frame_dims", self.ctx.h, C.byref(self.p), C.byref(M), C.byref(N))
        return M.value, N.value

    def set_init(self, U0):
        """U0 (2n, interleaved) for frame(init=INIT_GIVEN)."""
        a = _contig(U0) if _is_cuda(U0) else np.ascontiguousarray(U0, np.float64)
        call("aldic_set_init", self.ctx.h, _ptr(a), int(a.numel() if _is_cuda(a) else a.size))

    def set_init_gated(self, U0, F0=None, conf=None, conf_min=0.5):
        """An external guess for frame(init=INIT_GATED): U0 (2n), F0 (4n or
        None) and a confidence per node (n, float32, or None); nodes with
        conf >= conf_min start IC-GN from (U0, F0), the others from the
        integer search."""
        a = _contig(U0) if _is_cuda(U0) else np.ascontiguousarray(U0, np.float64)
        n = int(a.numel() if _is_cuda(a) else a.size) // 2
        fa = None if F0 is None else (_contig(F0) if _is_cuda(F0) else np.ascontiguousarray(F0, np.float64))
        ca = None if conf is None else (_contig(conf) if _is_cuda(conf)
                                        else np.ascontiguousarray(conf, np.float32))
        call("aldic_set_init_gated", self.ctx.h, _ptr(a), _ptr(fa), _ptr(ca), float(conf_min), n)

    def frame(self, out: dict | None = None, stats: bool = True, device_out: bool = False,
              init: int = INIT_SEARCH):
        """Run one frame.  With out (dict of preallocated arrays x0, y0, U, F,
        iters -- numpy or CUDA tensors) the results are written there.  init
        selects the initial guess (INIT_SEARCH, INIT_SEARCH_MG -- the
        multigrid search, which also decides the node grid -- or a sequence
        mode: INIT_PREV, INIT_ZERO, INIT_EXTRAP, INIT_GIVEN).  The sequence
        modes run on the grid of the last INIT_SEARCH_MG frame, if any since
        the last INIT_SEARCH frame."""
        self.p.init = int(init)
        mg = init == INIT_SEARCH_MG
        if init == INIT_SEARCH:
            self.node_grid = None
        for k in range(4):
            self.p.node_grid[k] = 0.0 if (mg or self.node_grid is None) else self.node_grid[k]
        if mg:
            if self.shape is None:
                raise AldicError("ALDIC.frame", -2, "set the reference image first")
            H, W = self.shape
            n = (W // self.p.step + 1) * (H // self.p.step + 1)   # capacity; the grid follows
            stats = True
        else:
            M, N = self.dims()
            n = M * N
        if out is None:
            if device_out:
                dev = torch.device("cuda", self.ctx.device)
                out = {"x0": torch.empty(n, dtype=torch.float64, device=dev),
                       "y0": torch.empty(n, dtype=torch.float64, device=dev),
                       "U": torch.empty(2 * n, dtype=torch.float64, device=dev),
                       "F": torch.empty(4 * n, dtype=torch.float64, device=dev),
                       "iters": torch.empty(n, dtype=torch.int32, device=dev)}
            else:
                out = {"x0": np.empty(n), "y0": np.empty(n), "U": np.empty(2 * n),
                       "F": np.empty(4 * n), "iters": np.empty(n, np.int32)}
        st = FrameStats()
        call("aldic_frame", self.ctx.h, C.byref(self.p), _ptr(out["x0"]), _ptr(out["y0"]),
             _ptr(out["U"]), _ptr(out["F"]), _ptr(out["iters"]), C.byref(st) if stats else None)
        res = dict(out)
        if mg:
            self.node_grid = tuple(st.node_grid)
            M, N = int(st.node_grid[2]), int(st.node_grid[3])
            n = M * N
            for k, m in (("x0", 1), ("y0", 1), ("U", 2), ("F", 4), ("iters", 1)):
                res[k] = out[k][:m * n]
        res["M"], res["N"] = M, N
        res["node_grid"] = tuple(st.node_grid) if stats else self.node_grid
        if stats:
            res["stats"] = {"beta": st.beta, "bad_icgn": st.bad_icgn,
                            "converged_icgn": st.converged_icgn,
                            "mean_iters_icgn": st.mean_iters_icgn,
                            "update_y": list(st.update_y)[:st.admm_steps],
                            "update_y2": list(st.update_y2)[:st.admm_steps],
                            "kernel_launches": st.kernel_launches,
                            "max_pcg_iters": st.max_pcg_iters,
                            "t_search_mg_ms": st.t_search_mg_ms,
                            "gated_init": st.gated_init,
                            "t_stage_ms": dict(zip(("normalize", "search", "icgn", "icgn_post",
                                                    "section5", "admm", "frame"),
                                                   list(st.t_stage_ms)[:7]))}
        return res


# ------------------------------------------------------------------ quadtree
class QuadtreeMesh:
    """The DICmesh of main_ALDIC_Quadtree.m (func_quadtree/GenerateQuadtreeMesh.m):
    coordinatesFEM (n x 2), elementsFEM (ne x 8, 1-based, slots 5-8 hanging
    nodes, 0 = none) and dirichlet (markCoordHoleEdge), held by the library
    (host data, device copies made on first use)."""

    def __init__(self, handle, owned=True):
        self.h = handle
        self.owned = owned   # False: a context's frame mesh, freed by the library
        n, ne, nd = C.c_int(), C.c_int(), C.c_int()
        call("aldic_qt_mesh_info", self.h, C.byref(n), C.byref(ne), C.byref(nd))
        self.n, self.ne, self.ndir = n.value, ne.value, nd.value
        c = np.empty((2, self.n))
        e = np.empty((8, self.ne), np.int32)
        d = np.empty(max(1, self.ndir), np.int32)
        call("aldic_qt_mesh_get", self.h, _ptr(c), _ptr(e), _ptr(d))
        self.coordinatesFEM = c.T.copy()
        self.elementsFEM = e.T.copy()
        self.dirichlet = d[:self.ndir].copy()

    @classmethod
    def generate(cls, coordinatesFEM, elementsFEM, mask, winstepsize, elementMinSize=2):
        """GenerateQuadtreeMesh.m on the uniform mesh of MeshSetUp (coordinates
        n x 2, elements ne x 4) and ImgRefMask (H, W) array."""
        c = np.asfortranarray(np.asarray(coordinatesFEM, np.float64))
        e = np.asfortranarray(np.asarray(elementsFEM, np.int32)[:, :4])
        m = np.ascontiguousarray(np.asarray(mask, np.float64))
        H, W = m.shape
        h = C.c_void_p()
        call("aldic_qt_mesh_generate", len(c), _ptr(c), len(e), _ptr(e), _ptr(m), W, H,
             float(winstepsize), int(elementMinSize), C.byref(h))
        return cls(h)

    @classmethod
    def create(cls, coordinatesFEM, elementsFEM, dirichlet):
        c = np.asfortranarray(np.asarray(coordinatesFEM, np.float64))
        e8 = np.zeros((len(elementsFEM), 8), np.int32)
        ea = np.asarray(elementsFEM, np.int32)
        e8[:, :ea.shape[1]] = ea
        e8 = np.asfortranarray(e8)
        d = np.ascontiguousarray(np.asarray(dirichlet, np.int32).reshape(-1))
        h = C.c_void_p()
        call("aldic_qt_mesh_create", len(c), _ptr(c), len(e8), _ptr(e8), len(d),
             _ptr(d) if len(d) else None, C.byref(h))
        return cls(h)

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "owned", True):
                _lib.lib().aldic_qt_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def GenerateQuadtreeMesh(DICmesh: dict, mask, winstepsize, elementMinSize=2) -> QuadtreeMesh:
    """func_quadtree/GenerateQuadtreeMesh.m:17-115 (the mesh part; U0 is
    interpolated separately)."""
    return QuadtreeMesh.generate(DICmesh["coordinatesFEM"], DICmesh["elementsFEM"], mask,
                                 winstepsize, elementMinSize)


def Subpb2Quadtree(mesh: QuadtreeMesh, beta, mu, U, F, ctx: Context | None = None):
    """func_quadtree/Subpb2Quadtree.m:1 (GaussPtOrder 2, alpha 0; the duals
    are multiplied by zero in the reference and are not taken)."""
    ctx = ctx or default_context()
    Ua, Fa = _prep(U), _prep(F)
    out = _empty(_first_cuda(Ua, Fa), (2 * mesh.n,))
    call("aldic_qt_subpb2", ctx.h, mesh.h, float(beta), float(mu), _ptr(Ua), _ptr(Fa), _ptr(out))
    return out


def funGlobalNodalStrainQuadtree(mesh: QuadtreeMesh, U, ctx: Context | None = None):
    """func_quadtree/funGlobalNodalStrainQuadtree.m:1 (nodal values by corner
    extrapolation and averaging; the reference interpolates scattered
    Gauss-point values)."""
    ctx = ctx or default_context()
    Ua = _prep(U)
    out = _empty(_first_cuda(Ua), (4 * mesh.n,))
    call("aldic_qt_nodal_strain", ctx.h, mesh.h, _ptr(Ua), _ptr(out))
    return out


def quadtree_fill(mesh: QuadtreeMesh, vals, bad, ctx: Context | None = None):
    """Refill of the flagged nodes of nf interleaved fields (n x nf)."""
    ctx = ctx or default_context()
    v = _prep(vals)
    v = v.clone() if _is_cuda(v) else v.copy()
    nf = (v.numel() if _is_cuda(v) else v.size) // mesh.n
    b = _prep(bad, np.uint8)
    call("aldic_qt_fill", ctx.h, mesh.h, int(nf), _ptr(v), _ptr(b))
    return v


def icgn_flags(iters, floor=float("nan"), ctx: Context | None = None):
    """Bad-subset flags on any node set (LocalICGN.m:117-131; floor 20 for
    Subpb1Quadtree.m:172-181): (bad mask, bad-point count)."""
    ctx = ctx or default_context()
    it = _prep(iters, np.int32)
    n = it.numel() if _is_cuda(it) else it.size
    bad = _empty(_first_cuda(it), (n,), np.uint8) if _is_cuda(it) else np.empty(n, np.uint8)
    nb = C.c_int()
    call("aldic_icgn_flags", ctx.h, int(n), _ptr(it), float(floor), _ptr(bad), C.byref(nb))
    return bad, nb.value


def _interp_uniform(xs, ys, fields, pts):
    # bilinear on the uniform node grid (stands in for scatteredInterpolant
    # 'linear' of GenerateQuadtreeMesh.m:124-130)
    x, y = pts[:, 0], pts[:, 1]
    i = np.clip(np.searchsorted(xs, x, side="right") - 1, 0, len(xs) - 2)
    j = np.clip(np.searchsorted(ys, y, side="right") - 1, 0, len(ys) - 2)
    tx = (x - xs[i]) / (xs[i + 1] - xs[i])
    ty = (y - ys[j]) / (ys[j + 1] - ys[j])
    return np.stack([(1 - ty) * ((1 - tx) * f[j, i] + tx * f[j, i + 1]) +
                     ty * ((1 - tx) * f[j + 1, i] + tx * f[j + 1, i + 1]) for f in fields], 1)


def quadtree_subset_sizes(mesh: QuadtreeMesh, winsize, mode="uniform", lo=16, hi=64):
    """Subset size per node: the reference's uniform winsize
    (Subpb1Quadtree.m:50), or ("element") twice the smallest side of the
    elements at the node, clipped to [lo, hi] and even."""
    c, E = mesh.coordinatesFEM, mesh.elementsFEM
    if mode == "uniform":
        return np.full(mesh.n, int(winsize), np.int32)
    if mode != "element":
        raise ValueError("subsets must be 'uniform' or 'element'")
    side = np.full(mesh.n, np.inf)
    sz = np.abs(c[E[:, 2] - 1, 0] - c[E[:, 0] - 1, 0])
    for k in range(8):
        nz = E[:, k] > 0
        np.minimum.at(side, E[nz, k] - 1, sz[nz])
    side[~np.isfinite(side)] = winsize / 2
    return (2 * np.round(np.clip(2 * side, lo, hi) / 2)).astype(np.int32)


def _select_beta(betas, e1, e2):
    # main_ALDIC_Quadtree.m:179-190
    e1, e2 = np.asarray(e1), np.asarray(e2)
    es = (e1 - e1.mean()) / e1.std(ddof=1) + (e2 - e2.mean()) / e2.std(ddof=1)
    k = int(np.nanargmin(es))
    if 1 <= k <= len(betas) - 2:
        p = np.polyfit(np.log10(betas[k - 1:k + 2]), es[k - 1:k + 2], 2)
        return 10 ** (-p[1] / 2 / p[0])
    return betas[k]


class ALDICQuadtree:
    """One frame of main_ALDIC_Quadtree.m Sections 3-6 (first frame of a
    sequence): integer search on the uniform grid and Init, the quadtree mesh
    of GenerateQuadtreeMesh.m with the initial guess interpolated onto it,
    LocalICGN on every quadtree node (+ flags and refill), the three-value
    beta sweep, Subpb2Quadtree + nodal strain with the boundary strains kept,
    then ADMM steps (Subpb1Quadtree, Subpb2Quadtree) until step 4 or an
    update below tol2.  Left out: the interactive outlier removal
    (funRemoveOutliersQuadtree) and the strain smoothing of
    DICpara.StrainSmoothness (regularizeNd).

        qt = ALDICQuadtree(winsize=32, step=16, search=16)
        qt.set_images(f, g, mask)     # mask: ImgRefMask as an (H, W) array
        res = qt.frame()              # coords, elems, U, F, ...
    """

    def __init__(self, winsize, step, search, tol=1e-2, mu=1e-3, n_admm=3, tol2=1e-2,
                 min_size=2, precision=FP32, subsets="uniform", device=None,
                 ctx: Context | None = None, gridx=None, gridy=None):
        self.ctx = ctx or default_context(device)
        self.w, self.step, self.search = int(winsize), int(step), int(search)
        self.gridx = None if gridx is None else (int(gridx[0]), int(gridx[-1]))
        self.gridy = None if gridy is None else (int(gridy[0]), int(gridy[-1]))
        self.tol, self.mu, self.n_admm, self.tol2 = float(tol), float(mu), int(n_admm), float(tol2)
        self.min_size, self.precision, self.subsets = int(min_size), int(precision), subsets
        self.mesh = None

    def set_images(self, f, g, mask):
        self.f, self.g = f, g
        self._mask_in = mask
        self.mask = np.ascontiguousarray(np.asarray(mask, np.float64))
        self._mask_key = None

    def frame(self):
        """One frame through aldic_qt_frame (all arrays on the device; the
        mesh is regenerated when the search grid or the mask changes)."""
        ctx = self.ctx
        f, g, mask = self.f, self.g, self.mask
        H, W = f.shape
        gx = self.gridx or (1, W)                 # DICpara.gridxyROIRange
        gy = self.gridy or (1, H)
        t0 = time.perf_counter()
        if self._mask_key != (id(self._mask_in), id(f), gx, gy):
            ctx.set_ref(f, roi=(gx[0], gx[1], gy[0], gy[1]), mask=mask)
            self._mask_key = (id(self._mask_in), id(f), gx, gy)
        ctx.set_def(g)
        p = QtFrameParams()
        p.winsize, p.step, p.search = self.w, self.step, self.search
        p.gridx[0], p.gridx[1] = gx
        p.gridy[0], p.gridy[1] = gy
        p.tol, p.mu, p.tol2, p.n_admm = self.tol, self.mu, self.tol2, self.n_admm
        p.min_size, p.precision = self.min_size, self.precision
        if self.subsets not in ("uniform", "element"):
            raise ValueError("subsets must be 'uniform' or 'element'")
        p.subsets = 1 if self.subsets == "element" else 0
        mh = C.c_void_p()
        st = QtFrameStats()
        call("aldic_qt_frame", ctx.h, C.byref(p), C.byref(mh), C.byref(st))
        if self.mesh is None or not st.mesh_reused:
            self.mesh = QuadtreeMesh(mh.value, owned=False)
        m = self.mesh
        n = st.n
        U0, Ui, U, F = np.empty(2 * n), np.empty(2 * n), np.empty(2 * n), np.empty(4 * n)
        it, wins = np.empty(n, np.int32), np.empty(n, np.int32)
        call("aldic_qt_frame_get", ctx.h, _ptr(U0), _ptr(Ui), _ptr(U), _ptr(F), _ptr(it), _ptr(wins))
        t1 = time.perf_counter()
        k = st.admm_steps
        tm = list(st.t_ms)
        return {"coords": m.coordinatesFEM, "elems": m.elementsFEM, "dirichlet": m.dirichlet,
                "U": U, "F": F, "U_icgn": Ui, "iters_icgn": it, "bad_icgn": st.bad_icgn,
                "beta": st.beta, "update_y": list(st.update_y)[:k],
                "update_y2": list(st.update_y2)[:k], "wins": wins, "U0": U0,
                "mesh_reused": bool(st.mesh_reused),
                "time_s": {"search": tm[0] / 1e3, "mesh": tm[1] / 1e3, "search_mesh": (tm[0] + tm[1]) / 1e3,
                           "icgn": tm[2] / 1e3, "section5": tm[3] / 1e3, "admm": tm[4] / 1e3,
                           "frame": t1 - t0}}


# ------------------------------------------------------------------ learned init
class InitNet:
    """The learned initial guess's network (aldic_cnn_*): 64 x 64 reference /
    deformed patch pairs -> [u/16, v/16, 20 du/dx, 20 dv/dx, 20 du/dy,
    20 dv/dy, confidence logit, 0], trained and run on the GPU by the
    library's own tcgen05 forward and backward kernels."""

    TSCALE, GSCALE = 16.0, 20.0

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        call("aldic_cnn_create", int(device), C.c_uint64(seed), C.byref(h))
        self.h, self.device = h, device
        self.n_params = int(_lib.lib().aldic_cnn_num_params())

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aldic_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        call("aldic_cnn_get_params", self.h, _ptr(p))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(np.asarray(p, np.float32))
        call("aldic_cnn_set_params", self.h, _ptr(p))

    def save(self, path):
        np.savez_compressed(path, params=self.get_params())

    def load(self, path):
        self.set_params(np.load(path)["params"])

    @staticmethod
    def _x(x):
        bf = _is_cuda(x) and x.dtype == torch.bfloat16
        return (x.contiguous() if _is_cuda(x) else np.ascontiguousarray(x, np.float32)), int(bf)

    def train_step(self, x, targets, lr, stream=None, grads=False, outputs=False):
        """One step on a batch; returns (loss, grads or None, outputs or None)."""
        xx, bf = self._x(x)
        B = xx.shape[0]
        t = targets.contiguous() if _is_cuda(targets) else np.ascontiguousarray(targets, np.float32)
        loss = C.c_double()
        g = np.empty(self.n_params, np.float32) if grads else None
        o = np.empty((B, 8), np.float32) if outputs else None
        sh = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        call("aldic_cnn_train_step", self.h, _ptr(xx), bf, _ptr(t), B, float(lr), C.c_void_p(sh),
             C.byref(loss), _ptr(g), _ptr(o))
        return loss.value, g, o

    def predict(self, x, stream=None, out=None):
        xx, bf = self._x(x)
        B = xx.shape[0]
        if out is None:
            out = (torch.empty((B, 8), dtype=torch.float32, device=xx.device) if _is_cuda(xx)
                   else np.empty((B, 8), np.float32))
        sh = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        call("aldic_cnn_predict", self.h, _ptr(xx), bf, B, C.c_void_p(sh), _ptr(out))
        return out


def cnn_patches(ctx: Context, coords, bf16=True):
    """64 x 64 normalised patch pairs around the nodes (coords n x 2) from the
    images set on ctx: a CUDA tensor n x 64 x 64 x 2."""
    cf = _coords_cm(coords)
    n = cf.shape[-1]
    out = torch.empty((n, 64, 64, 2), dtype=torch.bfloat16 if bf16 else torch.float32,
                      device=torch.device("cuda", ctx.device))
    call("aldic_cnn_patches", ctx.h, _ptr(cf), n, int(bf16), _ptr(out))
    return out


def cnn_to_init(ctx: Context, out):
    """U0 (2n), F0 (4n) and confidence (n) from network outputs (n x 8 CUDA
    tensor), on the device."""
    n = out.shape[0]
    dev = out.device
    U0 = torch.empty(2 * n, dtype=torch.float64, device=dev)
    F0 = torch.empty(4 * n, dtype=torch.float64, device=dev)
    conf = torch.empty(n, dtype=torch.float32, device=dev)
    call("aldic_cnn_to_init", ctx.h, _ptr(out.contiguous()), n, _ptr(U0), _ptr(F0), _ptr(conf))
    return U0, F0, conf


class ALDICSequence:
    """The frame loop of main_ALDIC.m:53-147 over an image sequence, with
    every image and all state on the device.

        seq = ALDICSequence(inc_unit=10, winsize=32, step=16, search=24)
        for res in seq.run(frames):      # frames[0] is the first reference
            ...

    Per frame ImgSeqNum = 2, 3, ... (1-based like the reference):
      * ImgSeqNum < 2 + n_search (the reference: < 7): integer search
        (NewFFTSearch = 1, main_ALDIC.m:69-75);
      * else, when mod(ImgSeqNum - 2, inc_unit) == 0 (incremental mode): the
        previous frame becomes the reference and U0 = 0 (main_ALDIC.m:118-126);
      * else U0 from earlier results: the previous U for the first frame after
        a reference change (main_ALDIC.m:130-131), later a constant-rate
        extrapolation from the last two frames solved against the same
        reference, standing in for the POD-GPR prediction of
        main_ALDIC.m:133-146 (predictor="previous" keeps the previous U).
    inc_unit=None is the accumulative mode (the reference never changes).
    Each yielded dict holds the frame's U, F, iters (CUDA tensors), its
    init mode, whether the reference was updated, and the device latency of
    the frame in ms (CUDA events around set_def + frame on the context
    stream)."""

    def __init__(self, inc_unit: int | None = None, n_search: int = 5, predictor: str = "extrap",
                 roi=None, mask=None, search_method: str = "whole", **frame_kw):
        if predictor not in ("extrap", "previous"):
            raise ValueError("predictor must be 'extrap' or 'previous'")
        if search_method not in ("whole", "multigrid"):
            raise ValueError("search_method must be 'whole' (InitFFTSearchMethod = 1) or "
                             "'multigrid' (funIntegerSearchMg)")
        self.search_mode = INIT_SEARCH if search_method == "whole" else INIT_SEARCH_MG
        self.al = ALDIC(**frame_kw)
        self.inc_unit = inc_unit
        self.n_search = max(1, int(n_search))
        self.predictor = predictor
        self.roi, self.mask = roi, mask

    def plan(self, n_frames: int):
        """(ImgSeqNum, init mode, reference frame index (0-based), update)
        for every deformed frame of an n_frames sequence."""
        out, ref, same = [], 0, 0
        for s in range(2, n_frames + 1):
            upd = False
            if s < 2 + self.n_search:
                mode = getattr(self, "search_mode", INIT_SEARCH)
            elif self.inc_unit and (s - 2) % self.inc_unit == 0:
                ref, upd, mode, same = s - 2, True, INIT_ZERO, 0
            elif self.predictor == "extrap" and same >= 2:
                mode = INIT_EXTRAP
            else:
                mode = INIT_PREV
            out.append((s, mode, ref, upd))
            same += 1
        return out

    def run(self, frames, stream=None):
        if torch is None or not torch.cuda.is_available():
            raise AldicError("ALDICSequence.run", -3, "a CUDA device is required")
        dev = torch.device("cuda", self.al.ctx.device)
        stream = stream or torch.cuda.Stream(dev)
        self.al.ctx.set_stream(stream)
        self.al.set_images(frames[0], roi=self.roi, mask=self.mask)
        for s, mode, ref, upd in self.plan(len(frames)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                if upd:
                    self.al.set_images(frames[ref], roi=self.roi, mask=self.mask)
                self.al.ctx.set_def(frames[s - 1])
                res = self.al.frame(device_out=True, init=mode, stats=False)
                e1.record(stream)
            e1.synchronize()
            res.update(img_seq_num=s, init=mode, ref_index=ref, ref_updated=upd,
                       latency_ms=e0.elapsed_time(e1))
            yield res

