"""The MEX gateways of 2d_aldic_b200/mex, built against the project's MEX
shim and driven exactly as MATLAB calls a MEX function.  The drop-in
ba_interp2 gateway must reproduce the reference's ba_interp2 (errors without
a GPU, results bit for bit with one)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")
SHIM = os.path.join(ROOT, "oracle", "mex_shim")
CLS = {np.dtype(np.float64): 6, np.dtype(np.float32): 7, np.dtype(np.int32): 12,
       np.dtype(np.uint8): 9, np.dtype(np.uint16): 11}


def build_gateway(src_name, out_name):
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, out_name)
    src = os.path.join(ROOT, "2d_aldic_b200", "mex", src_name)
    libdir = os.path.join(ROOT, "2d_aldic_b200")
    if not os.path.exists(out) or os.path.getmtime(out) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(libdir, "libaldic_b200.so"))):
        subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", f"-I{SHIM}",
                        f"-I{os.path.join(ROOT, 'include')}", "-o", out, src,
                        os.path.join(SHIM, "mex_shim.cpp"), os.path.join(SHIM, "mex_call.cpp"),
                        f"-L{libdir}", "-laldic_b200", f"-Wl,-rpath,{libdir}"], check=True)
    lib = C.CDLL(out)
    lib.shim_last_error.restype = C.c_char_p
    return lib


def mex_call(lib, nlhs, args, out_bytes):
    """Call mexFunction with numpy arrays (column-major MATLAB shapes given as
    the arrays' .T) or str (char arrays); returns (rc, outputs)."""
    cls, ndims, dims, datas, keep = [], [], [], [], []
    for a in args:
        if isinstance(a, str):
            arr = np.frombuffer(a.encode("utf-16-le"), dtype=np.uint16).copy()
            cls.append(4)
            d = [1, len(a)]
        else:
            arr = np.asfortranarray(np.atleast_2d(a) if np.ndim(a) < 2 else a)
            cls.append(CLS[arr.dtype])
            d = list(arr.shape)
        keep.append(arr)
        ndims.append(len(d))
        dims += d
        datas.append(arr.ctypes.data)
    outs = [np.zeros(b // 8 + 1, np.float64) for b in out_bytes]
    rc = lib.shim_call_mex_n(nlhs, len(args), (C.c_int * len(cls))(*cls),
                             (C.c_int * len(ndims))(*ndims), (C.c_longlong * len(dims))(*dims),
                             (C.c_void_p * len(datas))(*datas),
                             (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs]),
                             (C.c_size_t * len(out_bytes))(*out_bytes))
    return rc, outs


@pytest.fixture(scope="module")
def gw_interp():
    return build_gateway("ba_interp2_mex.cpp", "mex_ba_interp2.so")


@pytest.fixture(scope="module")
def gw_aldic():
    return build_gateway("aldic_mex.cpp", "mex_aldic.so")


def _ref_error(args, nlhs=1):
    import oracle
    ref = oracle.ref()
    ref.shim_last_error.restype = C.c_char_p
    rc, _ = mex_call(ref, nlhs, args, [8])
    return rc, ref.shim_last_error()


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference not compiled")
@pytest.mark.parametrize("case", ["nargs", "class", "size", "nlhs"])
def test_ba_interp2_gateway_errors_match_reference(gw_interp, case):
    F = np.random.default_rng(0).random((6, 5))
    X = np.ones((3, 1))
    if case == "nargs":
        args, nlhs = [F, X], 1
    elif case == "class":
        args, nlhs = [F, X.astype(np.float32), X], 1
    elif case == "size":
        args, nlhs = [F, X, np.ones((3, 1, 2))], 1
    else:
        args, nlhs = [F, X, X], 2
    rc, _ = mex_call(gw_interp, nlhs, args, [8, 8])
    rrc, rmsg = _ref_error(args, nlhs)
    assert rc == rrc == -1
    assert gw_interp.shim_last_error() == rmsg


def test_aldic_gateway_usage_errors(gw_aldic):
    rc, _ = mex_call(gw_aldic, 1, ["nosuch"], [8])
    assert rc == -1 and b"unknown command" in gw_aldic.shim_last_error()
    rc, _ = mex_call(gw_aldic, 1, ["icgn", np.zeros((2, 1))], [8])
    assert rc == -1 and b"icgn takes 8 arguments" in gw_aldic.shim_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_ba_interp2_gateway_matches_reference(gw_interp, dt):
    import oracle
    rng = np.random.default_rng(3)
    F = rng.uniform(0, 255, (40, 30, 2)).astype(dt)       # MATLAB M=40, N=30, P=2
    X = rng.uniform(-2, 33, (50, 7)).astype(dt)
    Y = rng.uniform(-2, 43, (50, 7)).astype(dt)
    rc, outs = mex_call(gw_interp, 1, [F, X, Y, "cubic"], [F.itemsize * X.size * 2])
    assert rc == 0
    got = outs[0].view(dt)[:X.size * 2]
    rref, ro = mex_call(oracle.ref(), 1, [F, X, Y], [F.itemsize * X.size * 2])
    assert rref == 0
    np.testing.assert_array_equal(got, ro[0].view(dt)[:X.size * 2])


@pytest.mark.gpu
def test_aldic_gateway_icgn_matches_oracle(gw_aldic, synth, oracle):
    W, H = 140, 120
    f = synth.speckle(W, H, 700, 31)
    g = synth.warp(f, synth.uniform_affine(0.002, -0.001, 0.4, -0.3), 0.5, 31)
    fn, _, _ = oracle.normalize(f)
    gn, _, _ = oracle.normalize(g)
    dx, dy = oracle.gradient(fn)
    xs = np.arange(30.0, 111.0, 10.0)
    X, Y = np.meshgrid(xs, np.arange(30.0, 91.0, 10.0))
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    n = len(coords)
    U0 = np.zeros(2 * n)
    # MATLAB orientation: images W x H column-major == numpy (H, W) C order -> pass .T
    args = ["icgn", U0[:, None], coords, dx[3:-3, 3:-3].T, dy[3:-3, 3:-3].T, fn.T, gn.T,
            np.array([[20.0]]), np.array([[1e-3]])]
    rc, outs = mex_call(gw_aldic, 4, args, [16 * n, 32 * n, 4 * n, 168 * n])
    assert rc == 0, gw_aldic.shim_last_error()
    U = outs[0][:2 * n]
    it = outs[2].view(np.int32)[:n]
    Uo, Fo, ito, Ho = oracle.icgn_batch(fn, gn, dx, dy, coords, U0, 20, 1e-3)
    np.testing.assert_array_equal(it, ito)
    np.testing.assert_allclose(U, Uo, atol=1e-8)


@pytest.mark.gpu
def test_aldic_gateway_searchmg_and_computestrain(gw_aldic, synth, oracle, aldic):
    """'searchmg' on the normalised images as MATLAB holds them equals the
    library's funIntegerSearchMg on the raw images (normalisation is affine,
    the correlation does not see it); 'computestrain' equals ComputeStrain."""
    W, H = 192, 160
    f = synth.speckle(W, H, 900, 33)
    g = synth.warp(f, synth.uniform_affine(0.004, -0.003, 14.6, -9.2), 2.0, 33)
    fn, _, _ = oracle.normalize(f)
    gn, _, _ = oracle.normalize(g)
    cap = (W // 8 + 1) * (H // 8 + 1)
    args = ["searchmg", fn.T, gn.T, np.array([[1.0, W]]), np.array([[1.0, H]]),
            np.array([[16.0]]), np.array([[8.0]])]
    rc, outs = mex_call(gw_aldic, 5, args, [8 * cap] * 5)
    assert rc == 0, gw_aldic.shim_last_error()
    x, y, u, v, cc = aldic.funIntegerSearchMg(f, g, [1, W], [1, H], 16, 8, 8)
    ny, nx = u.shape
    for got, ref in zip(outs, (x, y, u, v, cc["max"])):
        m = got[:nx * ny].reshape(nx, ny).T                 # MATLAB ny x nx column-major
        np.testing.assert_allclose(m, ref, rtol=0, atol=1e-6)
    # ComputeStrain, plane fitting, Green-Lagrangian
    M, N = nx, ny
    U = np.empty(2 * M * N)
    U[0::2], U[1::2] = u.reshape(-1), v.reshape(-1)
    args = ["computestrain", np.array([[float(M)]]), np.array([[float(N)]]), np.array([[8.0]]),
            np.array([[2.0]]), np.array([[2.0]]), np.array([[2.0]]), U[:, None], np.zeros((0, 0))]
    rc, outs = mex_call(gw_aldic, 2, args, [32 * M * N, 32 * M * N])
    assert rc == 0, gw_aldic.shim_last_error()
    r = aldic.ComputeStrain(U, None, {"M": M, "N": N},
                            {"MethodToComputeStrain": 2, "StrainType": 2, "PlaneFitRad": 2,
                             "winstepsize": 8})
    np.testing.assert_array_equal(outs[0][:4 * M * N], r["FStrain"])
    np.testing.assert_array_equal(outs[1][:4 * M * N], r["FStrainFinite"])


def test_aldic_gateway_new_command_usage(gw_aldic):
    for cmd, msg in (("intsearch", b"intsearch takes 7 arguments"),
                     ("subpb2qt", b"subpb2qt takes 7 arguments"),
                     ("frame", b"frame takes 11 arguments")):
        rc, _ = mex_call(gw_aldic, 1, [cmd, np.zeros((2, 1))], [8])
        assert rc == -1 and msg in gw_aldic.shim_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uint8", "double"])
def test_aldic_gateway_intsearch_matches_oracle(gw_aldic, synth, oracle, kind):
    """funIntegerSearch through the gateway as IntegerSearch.m:54 calls it:
    [x,y,u,v,cc] = funIntegerSearch(f,g,searchSize,gridx,gridy,winsize,step,0,step)
    -- on raw 8-bit images (exact integer correlation) and on the normalised
    doubles MATLAB passes; peaks equal the oracle's."""
    W, H = 200, 170
    f = synth.speckle(W, H, 1100, 41)
    g = synth.warp(f, synth.uniform_affine(0.003, -0.002, 2.6, -1.7), 2.0, 41)
    roi = (11, 190, 6, 161)
    if kind == "uint8":
        fa, ga = f.T, g.T
    else:
        fa, ga = oracle.normalize(f, roi)[0].T, oracle.normalize(g, roi)[0].T
    args = ["intsearch", fa, ga, np.array([[6.0, 6.0]]), np.array([[11.0, 190.0]]),
            np.array([[6.0, 161.0]]), np.array([[20.0]]), np.array([[10.0]])]
    nx, ny, _, _ = oracle.search_dims(W, H, (11, 190), (6, 161), 20, 10, (6, 6))
    n = nx * ny
    rc, outs = mex_call(gw_aldic, 6, args, [8 * n] * 5 + [16 * n])
    assert rc == 0, gw_aldic.shim_last_error()
    mg = oracle.normalize(g, roi)[1]
    xo, yo, uo, vo, co, qo = oracle.int_search(f, g, mg, (11, 190), (6, 161), 20, 10, (6, 6), True)
    for got, ref in zip(outs[:5], (xo, yo, uo, vo, co)):
        m = got[:n].reshape(nx, ny).T                        # ny x nx column-major
        if kind == "uint8":
            np.testing.assert_array_equal(m, ref)
        else:
            np.testing.assert_allclose(m, ref, rtol=0, atol=1e-9)
    q = outs[5][:2 * n].reshape(2, n).T
    qo = np.asarray(qo)
    np.testing.assert_allclose(q, qo.T if qo.shape[0] == 2 else qo, rtol=1e-9, equal_nan=True)


@pytest.mark.gpu
def test_aldic_gateway_subpb2qt_matches_oracle(gw_aldic, oracle):
    """Subpb2Quadtree.m through the gateway on the reference's own Sample12
    mesh (MATLAB's column-major DICmesh arrays) against the oracle's sparse
    direct restatement."""
    from oracle import quadtree as Q
    from test_reference_pins import sample12
    z = sample12()
    c, E, d = z["coordinatesFEM"], z["elementsFEM"], z["dirichlet"]
    n = len(c)
    rng = np.random.default_rng(5)
    U = rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    beta, mu = 2.56e-4, 1e-3
    args = ["subpb2qt", c, E.astype(np.float64), d.astype(np.float64)[:, None], np.array([[beta]]),
            np.array([[mu]]), U[:, None], F[:, None]]
    rc, outs = mex_call(gw_aldic, 1, args, [16 * n])
    assert rc == 0, gw_aldic.shim_last_error()
    ref = Q.subpb2_quadtree(c, E, d, beta, mu, U, F)
    np.testing.assert_allclose(outs[0][:2 * n], ref, rtol=1e-8, atol=1e-9)


@pytest.mark.gpu
def test_aldic_gateway_frame_matches_oracle(gw_aldic, synth, oracle):
    """The whole frame (main_ALDIC.m Sections 3-6) through the gateway on raw
    8-bit images: the FP64 oracle frame within 1e-4 px, the mesh exact."""
    wl = synth.workload("plain512", scale_down=2)
    f, g = wl.images()
    H, W = f.shape
    args = ["frame", f.T, g.T, np.array([[float(wl.winsize)]]), np.array([[float(wl.step)]]),
            np.array([[float(wl.search)]]), np.array([[1.0, W]]), np.array([[1.0, H]]),
            np.array([[wl.tol]]), np.array([[2.0]]), np.array([[2.0]]), np.array([[0.0]])]
    nx, ny, _, _ = oracle.search_dims(W, H, (1, W), (1, H), wl.winsize, wl.step,
                                      (wl.search, wl.search))
    n = nx * ny
    rc, outs = mex_call(gw_aldic, 6, args, [8 * n, 8 * n, 16 * n, 32 * n, 4 * n, 8 * 8])
    assert rc == 0, gw_aldic.shim_last_error()
    ro = oracle.frame(f, g, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=2)
    np.testing.assert_array_equal(outs[0][:n], ro["x0"])
    np.testing.assert_array_equal(outs[1][:n], ro["y0"])
    assert np.abs(outs[2][:2 * n] - ro["U"]).max() < 1e-4
    assert abs(outs[5][0] - ro["beta"]) < 1e-9 * ro["beta"]
