"""Python bindings of the CPU oracle (liboracle.so) and of the reference's own
compiled ba_interp2 (oracle/_ref/libba_interp2_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline / reference arm.  The product package never imports
this module.

Array conventions follow the reference after ReadImage's transpose: an image
is W x H with Img(x, y) and x fastest, i.e. a numpy array of shape (H, W);
node order is x-fastest; U is interleaved [u1 v1 u2 v2 ...]; F is
[F11 F21 F12 F22] per node; H21 is n x 21 column-major (numpy shape (21, n)).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libba_interp2_ref.so")

_DT = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2,
       np.dtype(np.float64): 3}


def build(ref_dir: str | None = None) -> None:
    """Compile the oracle (and the reference interpolator if its sources are
    present) with oracle/Makefile."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_dir:
        cmd.append(f"REF={ref_dir}")
    subprocess.run(cmd, check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _setup(_lib)
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(_REF)
        _ref.shim_call_mex.restype = C.c_int
    return _ref


P = C.c_void_p
I64 = C.c_int64


def _setup(L):
    L.orc_ba_interp2_f64.argtypes = [P, I64, I64, I64, P, P, I64, P]
    L.orc_ba_interp2_f32.argtypes = [P, I64, I64, I64, P, P, I64, P]
    L.orc_normalize.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P, P, P]
    L.orc_gradient.argtypes = [P, P, C.c_int, C.c_int, P, P]
    L.orc_search_dims.argtypes = [C.c_int, C.c_int, P, P, C.c_int, C.c_int, P, P, P, P, P]
    L.orc_int_search.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_double, P, P, C.c_int,
                                 C.c_int, P, P, P, P, P, P, P]
    L.orc_icgn_batch.argtypes = [P, P, P, P, C.c_int, C.c_int, P, I64, P, P, C.c_int,
                                 C.c_double, P, P, P, P]
    L.orc_subpb1_batch.argtypes = [P, P, P, P, C.c_int, C.c_int, P, I64, P, P, P, P, P,
                                   C.c_int, C.c_double, C.c_double, P, P]
    L.orc_localicgn_post.argtypes = [C.c_int, C.c_int, P, P, P]
    L.orc_subpb1_post.argtypes = [C.c_int, C.c_int, P, P]
    L.orc_gridfit_springs.argtypes = [C.c_int, C.c_int, C.c_int, P, P]
    L.orc_inpaint_springs.argtypes = [C.c_int, C.c_int, P]
    L.orc_subpb2.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, P, P, P,
                             P, P]
    L.orc_nodal_strain.argtypes = [C.c_int, C.c_int, C.c_double, P, P]
    L.orc_smooth_fields.argtypes = [C.c_int, C.c_int, C.c_int, P]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    L.orc_frame.argtypes = [P, P, C.c_int, C.c_int, C.c_int, P, P]
    L.orc_frame_free.argtypes = [P]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _c(a, dt=None):
    a = np.asarray(a)
    if dt is not None:
        a = a.astype(dt, copy=False)
    return np.ascontiguousarray(a)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return lib().orc_get_threads()


# ---------------------------------------------------------------- a3
def ba_interp2(F, X, Y):
    """Z = ba_interp2(F, X, Y): F given MATLAB-style as a column-major M x N
    (x P) array -- pass a numpy array of shape (N, M) or (P, N, M) in C order
    (equivalently F.T of the MATLAB matrix)."""
    F = np.asarray(F)
    dt = np.float64 if F.dtype == np.float64 else np.float32
    F = _c(F, dt)
    if F.ndim == 2:
        Pn, N, M = 1, F.shape[0], F.shape[1]
    else:
        Pn, N, M = F.shape
    X = _c(X, dt)
    Y = _c(Y, dt)
    n = X.size
    out = np.empty((Pn,) + X.shape, dt)
    fn = lib().orc_ba_interp2_f64 if dt == np.float64 else lib().orc_ba_interp2_f32
    fn(_p(F), M, N, Pn, _p(X), _p(Y), n, _p(out))
    return out[0] if Pn == 1 else out


def ref_ba_interp2(F, X, Y):
    """The reference's own ba_interp2.cpp (compiled into oracle/_ref), driven
    through its mexFunction exactly as MATLAB would call it."""
    F = np.asarray(F)
    dt = np.float64 if F.dtype == np.float64 else np.float32
    cls = 6 if dt == np.float64 else 7
    F = _c(F, dt)
    X = _c(X, dt)
    Y = _c(Y, dt)
    if F.ndim == 2:
        fd = [F.shape[1], F.shape[0]]
    else:
        fd = [F.shape[2], F.shape[1], F.shape[0]]
    xd = [X.size, 1]
    Pn = 1 if F.ndim == 2 else F.shape[0]
    out = np.empty(X.size * Pn, dt)
    dims = (C.c_longlong * 16)(*(fd + xd + xd))
    ndims = (C.c_int * 3)(len(fd), 2, 2)
    clss = (C.c_int * 3)(cls, cls, cls)
    datas = (C.c_void_p * 3)(F.ctypes.data, X.ctypes.data, Y.ctypes.data)
    od = (C.c_longlong * 8)()
    ond = C.c_int(0)
    rc = ref().shim_call_mex(1, 3, clss, ndims, dims, datas, out.ctypes.data,
                             C.c_size_t(out.nbytes), od, C.byref(ond))
    if rc != 0:
        raise RuntimeError(f"reference ba_interp2 failed ({rc})")
    return out.reshape((Pn,) + X.shape) if Pn > 1 else out.reshape(X.shape)


# ---------------------------------------------------------------- a1/a2
def normalize(img, roi=None):
    img = np.asarray(img)
    H, W = img.shape
    img = _c(img)
    dt = _DT[img.dtype]
    roi = np.asarray(roi if roi is not None else [1, W, 1, H], np.int32)
    out = np.empty((H, W), np.float64)
    m = C.c_double()
    s = C.c_double()
    rc = lib().orc_normalize(_p(img), dt, W, H, _p(roi), _p(out), C.byref(m), C.byref(s))
    if rc:
        raise ValueError("empty ROI")
    return out, m.value, s.value


def gradient(f, mask=None):
    f = _c(f, np.float64)
    H, W = f.shape
    dx = np.empty_like(f)
    dy = np.empty_like(f)
    m = _c(mask, np.float64) if mask is not None else None
    lib().orc_gradient(_p(f), _p(m), W, H, _p(dx), _p(dy))
    return dx, dy


# ---------------------------------------------------------------- a4/a5
def search_dims(W, H, gridx, gridy, winsize, step, search):
    gx = np.asarray(gridx, np.int32)
    gy = np.asarray(gridy, np.int32)
    s = np.asarray(search, np.int32)
    nx, ny, x1, y1 = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rc = lib().orc_search_dims(W, H, _p(gx), _p(gy), winsize, step, _p(s), C.byref(nx),
                               C.byref(ny), C.byref(x1), C.byref(y1))
    if rc:
        raise ValueError("bad search parameters")
    return nx.value, ny.value, x1.value, y1.value


def int_search(f_raw, g_raw, mu_g, gridx, gridy, winsize, step, search, qfactors=False):
    """funIntegerSearch whole-field core; returns x, y, u, v, ccmax (ny x nx)
    and qfactors (n x 2) or None."""
    f_raw = _c(f_raw)
    g_raw = _c(g_raw, f_raw.dtype)
    H, W = f_raw.shape
    nx, ny, _, _ = search_dims(W, H, gridx, gridy, winsize, step, search)
    outs = [np.empty((nx, ny), np.float64) for _ in range(5)]  # column-major ny x nx
    q = np.empty((2, nx * ny), np.float64) if qfactors else None
    gx = np.asarray(gridx, np.int32)
    gy = np.asarray(gridy, np.int32)
    s = np.asarray(search, np.int32)
    rc = lib().orc_int_search(_p(f_raw), _p(g_raw), _DT[f_raw.dtype], W, H, float(mu_g),
                              _p(gx), _p(gy), winsize, step, _p(s), *[_p(o) for o in outs],
                              _p(q))
    if rc:
        raise ValueError("search failed")
    res = [o.T for o in outs]  # (ny, nx) MATLAB orientation
    return (*res, (q.T if q is not None else None))


# ---------------------------------------------------------------- a7-a9
def icgn_batch(f, g, dfdx, dfdy, coords, U0, winsize, tol):
    f, g, dfdx, dfdy = (_c(a, np.float64) for a in (f, g, dfdx, dfdy))
    H, W = f.shape
    coords = np.asfortranarray(np.asarray(coords, np.float64).reshape(-1, 2))
    n = coords.shape[0]
    U0 = _c(U0, np.float64)
    U = np.empty(2 * n)
    F = np.empty(4 * n)
    it = np.empty(n, np.int32)
    H21 = np.empty((21, n))
    wa = None
    w = winsize
    if np.ndim(winsize) > 0:
        wa = _c(winsize, np.int32)
        w = 0
    lib().orc_icgn_batch(_p(f), _p(g), _p(dfdx), _p(dfdy), W, H, _p(np.ravel(coords, "F")), n,
                         _p(U0), _p(wa), int(w), float(tol), _p(U), _p(F), _p(it), _p(H21))
    return U, F, it, H21


def subpb1_batch(f, g, dfdx, dfdy, coords, UOld, FOld, vdual, H21, winsize, mu, tol):
    f, g, dfdx, dfdy = (_c(a, np.float64) for a in (f, g, dfdx, dfdy))
    H, W = f.shape
    coords = np.asarray(coords, np.float64).reshape(-1, 2)
    n = coords.shape[0]
    cf = np.ravel(coords, "F").copy()
    U = np.empty(2 * n)
    it = np.empty(n, np.int32)
    wa = None
    w = winsize
    if np.ndim(winsize) > 0:
        wa = _c(winsize, np.int32)
        w = 0
    H21 = _c(H21, np.float64)
    lib().orc_subpb1_batch(_p(f), _p(g), _p(dfdx), _p(dfdy), W, H, _p(cf), n,
                           _p(_c(UOld, np.float64)), _p(_c(FOld, np.float64)),
                           _p(_c(vdual, np.float64)), _p(H21), _p(wa), int(w), float(mu),
                           float(tol), _p(U), _p(it))
    return U, it


def localicgn_post(M, N, iters, U, F):
    U = _c(U, np.float64).copy()
    F = _c(F, np.float64).copy()
    nb = lib().orc_localicgn_post(M, N, _p(_c(iters, np.int32)), _p(U), _p(F))
    return U, F, nb


def subpb1_post(M, N, iters, U):
    U = _c(U, np.float64).copy()
    nb = lib().orc_subpb1_post(M, N, _p(_c(iters, np.int32)), _p(U))
    return U, nb


def gridfit_springs(M, N, fields):
    a = _c(fields, np.float64).reshape(-1, M * N).copy()
    rc = lib().orc_gridfit_springs(M, N, a.shape[0], _p(a), _p(a))
    if rc < 0:
        raise ValueError("gridfit: insufficient data")
    return a


def inpaint_springs(M, N, z):
    z = _c(z, np.float64).copy()
    lib().orc_inpaint_springs(M, N, _p(z))
    return z


def subpb2(M, N, step, beta, mu, U, F, udual, vdual):
    out = np.empty(2 * M * N)
    it = lib().orc_subpb2(M, N, float(step), float(beta), float(mu), _p(_c(U, np.float64)),
                          _p(_c(F, np.float64)), _p(_c(udual, np.float64)),
                          _p(_c(vdual, np.float64)), _p(out))
    return out, it


def nodal_strain(M, N, step, U):
    out = np.empty(4 * M * N)
    lib().orc_nodal_strain(M, N, float(step), _p(_c(U, np.float64)), _p(out))
    return out


def smooth_fields(M, N, vals, nf):
    v = _c(vals, np.float64).copy()
    if lib().orc_smooth_fields(M, N, nf, _p(v)):
        raise ValueError("smoothing failed")
    return v


# ---------------------------------------------------------------- a12
class _FP(C.Structure):
    _fields_ = [("winsize", C.c_int), ("step", C.c_int), ("search", C.c_int * 2),
                ("gridx", C.c_int * 2), ("gridy", C.c_int * 2), ("tol", C.c_double),
                ("mu", C.c_double), ("beta", C.c_double), ("n_admm", C.c_int),
                ("tol2", C.c_double), ("smooth", C.c_int),
                ("init_U", C.POINTER(C.c_double))]


class _FR(C.Structure):
    _fields_ = [("M", C.c_int), ("N", C.c_int), ("x0", C.POINTER(C.c_double)),
                ("y0", C.POINTER(C.c_double)), ("U", C.POINTER(C.c_double)),
                ("F", C.POINTER(C.c_double)), ("U_icgn", C.POINTER(C.c_double)),
                ("F_icgn", C.POINTER(C.c_double)), ("iters_icgn", C.POINTER(C.c_int32)),
                ("beta", C.c_double), ("admm_steps", C.c_int),
                ("update_y", C.c_double * 16), ("update_y2", C.c_double * 16),
                ("t_search", C.c_double), ("t_icgn", C.c_double), ("t_subpb1", C.c_double),
                ("t_subpb2", C.c_double), ("t_total", C.c_double)]


def frame(f_raw, g_raw, winsize, step, search, gridx=None, gridy=None, tol=1e-2, mu=1e-3,
          beta=0.0, n_admm=3, tol2=0.0, smooth=False, U0=None):
    """One frame of the ADMM core (main_ALDIC.m Sections 3-6); U0 (2n) replaces
    the integer search and Init for a later frame of a sequence."""
    f_raw = _c(f_raw)
    g_raw = _c(g_raw, f_raw.dtype)
    H, W = f_raw.shape
    p = _FP()
    p.winsize, p.step = winsize, step
    p.search[0], p.search[1] = (search, search) if np.ndim(search) == 0 else search
    gx = gridx or (1, W)
    gy = gridy or (1, H)
    p.gridx[0], p.gridx[1] = gx
    p.gridy[0], p.gridy[1] = gy
    p.tol, p.mu, p.beta, p.n_admm, p.tol2, p.smooth = tol, mu, beta, n_admm, tol2, int(smooth)
    if U0 is not None:
        U0 = np.ascontiguousarray(U0, np.float64)
        p.init_U = U0.ctypes.data_as(C.POINTER(C.c_double))
    r = _FR()
    rc = lib().orc_frame(_p(f_raw), _p(g_raw), _DT[f_raw.dtype], W, H, C.byref(p), C.byref(r))
    if rc:
        raise RuntimeError("oracle frame failed")
    n = r.M * r.N

    def arr(ptr, k, dt=np.float64):
        return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dt, copy=True)

    out = dict(M=r.M, N=r.N, x0=arr(r.x0, n), y0=arr(r.y0, n), U=arr(r.U, 2 * n),
               F=arr(r.F, 4 * n), U_icgn=arr(r.U_icgn, 2 * n), F_icgn=arr(r.F_icgn, 4 * n),
               iters_icgn=arr(r.iters_icgn, n, np.int32), beta=r.beta,
               admm_steps=r.admm_steps, update_y=list(r.update_y)[:r.admm_steps],
               update_y2=list(r.update_y2)[:r.admm_steps], t_search=r.t_search,
               t_icgn=r.t_icgn, t_subpb1=r.t_subpb1, t_subpb2=r.t_subpb2, t_total=r.t_total)
    lib().orc_frame_free(C.byref(r))
    return out
