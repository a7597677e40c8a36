"""Quadtree global step on the GPU against the oracle: Subpb2Quadtree.m
(hanging-node shape functions, Dirichlet nodes), the quadtree nodal strain
and the refill of flagged nodes, on a plate-with-hole mesh."""
import numpy as np
import pytest

from oracle import quadtree as Q

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plate(aldic):
    W = H = 512
    step = 16
    xs = np.arange(41, W - 56, step) + 16.0
    X, Y = np.meshgrid(xs, xs)
    coords, el = Q.uniform_mesh(X.reshape(-1), Y.reshape(-1), len(xs), len(xs))
    yy, xx = np.mgrid[1:H + 1, 1:W + 1]
    mask = ((xx - 256.0) ** 2 + (yy - 256.0) ** 2 >= 75 ** 2).astype(np.float64)
    c, E, d = Q.generate_quadtree_mesh(coords, el, mask, step)
    m = aldic.QuadtreeMesh.create(c, E, d)
    return c, E, d, m


def _fields(c, seed=0):
    rng = np.random.default_rng(seed)
    x, y = c[:, 0], c[:, 1]
    u = 0.3 + 0.002 * x + 0.5 * np.sin(2 * np.pi * y / 300) + 0.01 * rng.standard_normal(len(x))
    v = -0.2 - 0.001 * y + 0.3 * np.cos(2 * np.pi * x / 250) + 0.01 * rng.standard_normal(len(x))
    U = np.empty(2 * len(x))
    U[0::2], U[1::2] = u, v
    F = np.empty(4 * len(x))
    F[0::4] = 0.002 + 1e-3 * rng.standard_normal(len(x))
    F[1::4] = 0.5 * 2 * np.pi / 300 * np.cos(2 * np.pi * y / 300)
    F[2::4] = -0.3 * 2 * np.pi / 250 * np.sin(2 * np.pi * x / 250)
    F[3::4] = -0.001 + 1e-3 * rng.standard_normal(len(x))
    return U, F


@pytest.mark.parametrize("beta", [1e-3 * 256 * 1e-3, 1e-1 * 256 * 1e-3])
def test_qt_subpb2_matches_oracle(aldic, plate, beta):
    c, E, d, m = plate
    U, F = _fields(c)
    mu = 1e-3
    ref = Q.subpb2_quadtree(c, E, d, beta, mu, U, F)
    out = aldic.Subpb2Quadtree(m, beta, mu, U, F)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-8)
    # Dirichlet nodes keep U, nodes in no element get 0
    dd = d - 1
    np.testing.assert_array_equal(out[2 * dd], U[2 * dd])
    np.testing.assert_array_equal(out[2 * dd + 1], U[2 * dd + 1])
    involved = np.zeros(len(c), bool)
    involved[E[E > 0] - 1] = True
    assert not out[0::2][~involved].any()


def test_qt_strain_matches_oracle(aldic, plate):
    c, E, d, m = plate
    U, _ = _fields(c, 1)
    ref = Q.nodal_strain_quadtree(c, E, U)
    out = aldic.funGlobalNodalStrainQuadtree(m, U)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)
    # an affine field gives its gradient exactly, in the reference's slot order
    x, y = c[:, 0], c[:, 1]
    Ua = np.empty(2 * len(x))
    Ua[0::2] = 1.0 + 0.01 * x - 0.02 * y
    Ua[1::2] = -2.0 + 0.03 * x + 0.005 * y
    Fa = aldic.funGlobalNodalStrainQuadtree(m, Ua).reshape(-1, 4)
    involved = np.zeros(len(c), bool)
    involved[E[:, :4].reshape(-1) - 1] = True
    np.testing.assert_allclose(Fa[involved], np.tile([0.01, -0.02, 0.03, 0.005], (involved.sum(), 1)),
                               atol=1e-12)


def test_qt_fill_matches_oracle(aldic, plate):
    c, E, d, m = plate
    rng = np.random.default_rng(3)
    n = len(c)
    vals = np.stack([np.sin(c[:, 0] / 40.0), np.cos(c[:, 1] / 50.0), c[:, 0] * 1e-3], 1)
    bad = rng.random(n) < 0.1
    vin = vals.copy()
    vin[bad] = np.nan
    ref = Q.graph_fill(n, Q.mesh_edges(E), np.where(bad[:, None], 0.0, vin), bad)
    out = aldic.quadtree_fill(m, np.where(bad[:, None], 0.0, vin), bad.astype(np.uint8)).reshape(n, 3)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-8)
    np.testing.assert_array_equal(out[~bad], vals[~bad])
    inv = np.zeros(n, bool)
    inv[E[E > 0] - 1] = True
    # refilled values of mesh nodes follow the smooth field
    err = np.abs(out[bad & inv] - vals[bad & inv])
    assert np.median(err) < 0.01 and err.max() < 0.25


@pytest.fixture(scope="module")
def plate_images(synth):
    wl = synth.workload("plate2048", scale_down=4)       # 512^2, hole r = 75
    f, g = wl.images()
    return wl, f, g, wl.mask()


def test_quadtree_frame_fp64_matches_oracle(aldic, plate_images):
    wl, f, g, mask = plate_images
    ro = Q.frame(f, g, mask, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3)
    qt = aldic.ALDICQuadtree(wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3,
                             precision=aldic.FP64)
    qt.set_images(f, g, mask)
    r = qt.frame()
    np.testing.assert_array_equal(r["coords"], ro["coords"])
    np.testing.assert_array_equal(r["elems"], ro["elems"])
    np.testing.assert_array_equal(r["dirichlet"], ro["dirichlet"])
    np.testing.assert_allclose(r["U0"], ro["U0"], atol=1e-12)
    assert (r["iters_icgn"] == ro["iters_icgn"]).mean() > 0.995
    assert r["beta"] == pytest.approx(ro["beta"], rel=1e-6)
    assert len(r["update_y"]) == len(ro["update_y"])
    assert np.abs(r["U"] - ro["U"]).max() < 1e-4
    assert np.abs(r["F"] - ro["F"]).max() < 1e-4
    # accuracy against the plate-with-hole field at the nodes of the mesh
    c = r["coords"]
    inv = np.zeros(len(c), bool)
    inv[r["elems"][r["elems"] > 0] - 1] = True
    ut, vt = wl.field(c[:, 0], c[:, 1])
    e = np.r_[(r["U"][0::2] - ut)[inv], (r["U"][1::2] - vt)[inv]]
    assert np.sqrt(np.mean(e ** 2)) < 0.1


def test_quadtree_frame_element_sized_subsets(aldic, plate_images):
    wl, f, g, mask = plate_images
    qt = aldic.ALDICQuadtree(wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3,
                             subsets="element")
    qt.set_images(f, g, mask)
    r = qt.frame()
    assert set(np.unique(r["wins"])) <= {16, 32, 64} and r["wins"].min() == 16
    ro = Q.frame(f, g, mask, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3,
                 subsets="element")
    np.testing.assert_array_equal(r["wins"], ro["wins"])
    # FP32 sampling against the FP64 oracle: <= 0.01 px RMS on the mesh nodes
    inv = np.zeros(len(r["coords"]), bool)
    inv[r["elems"][r["elems"] > 0] - 1] = True
    d = (r["U"] - ro["U"]).reshape(-1, 2)[inv]
    assert np.sqrt(np.mean(d ** 2)) < 0.01
