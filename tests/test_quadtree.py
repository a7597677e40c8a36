"""Quadtree meshes (func_quadtree/GenerateQuadtreeMesh.m, QrefineR.m): the
library's host-side generator against the oracle's restatement, node for
node and element for element, plus the structural rules of the reference's
refinement.  CPU only (no device work)."""
import numpy as np
import pytest

from oracle import quadtree as Q


def _uniform(W, H, step, w, search):
    lo = 1 + search + w // 2
    xs = np.arange(lo, W - w - search - step, step) + w / 2
    ys = np.arange(lo, H - w - search - step, step) + w / 2
    X, Y = np.meshgrid(xs, ys)
    return Q.uniform_mesh(X.reshape(-1), Y.reshape(-1), len(xs), len(ys))


def _holes(W, H, holes):
    yy, xx = np.mgrid[1:H + 1, 1:W + 1]
    m = np.ones((H, W))
    for cx, cy, r in holes:
        m[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = 0.0
    return m


CASES = [
    # (W, H, step, holes, min_size)
    (512, 512, 16, [(256, 256, 75)], 2),
    (640, 384, 16, [(200, 190, 60), (470, 170, 45)], 2),
    (512, 512, 8, [(300.5, 240.25, 90)], 2),
    (768, 768, 32, [(384, 384, 150)], 4),
]


@pytest.mark.parametrize("W,H,step,holes,min_size", CASES)
def test_mesh_matches_oracle(aldic, W, H, step, holes, min_size):
    coords, el = _uniform(W, H, step, 32, 16)
    mask = _holes(W, H, holes)
    c, E, d = Q.generate_quadtree_mesh(coords, el, mask, step, min_size)
    m = aldic.QuadtreeMesh.generate(coords, el, mask, step, min_size)
    assert (m.n, m.ne, m.ndir) == (len(c), len(E), len(d))
    np.testing.assert_array_equal(m.coordinatesFEM, c)
    np.testing.assert_array_equal(m.elementsFEM, E)
    np.testing.assert_array_equal(m.dirichlet, d)
    # structure: the uniform nodes come first and keep their numbers
    np.testing.assert_array_equal(c[:len(coords)], coords)
    sizes = np.abs(c[E[:, 2] - 1, 0] - c[E[:, 0] - 1, 0])
    assert sizes.min() <= 2 * min_size and sizes.max() == step
    # elements are squares (corners 1..4 around the boundary)
    p = c[E[:, :4] - 1]
    area = 0.5 * np.sum(p[:, :, 0] * np.roll(p[:, :, 1], -1, 1) - np.roll(p[:, :, 0], -1, 1) * p[:, :, 1], 1)
    np.testing.assert_allclose(np.abs(area), sizes ** 2)
    # every hanging node sits at the midpoint of its element's edge
    for slot, (a, b) in zip(range(4, 8), [(1, 2), (2, 3), (3, 0), (0, 1)]):
        k = np.nonzero(E[:, slot])[0]
        mid = (c[E[k, a] - 1] + c[E[k, b] - 1]) / 2
        np.testing.assert_array_equal(c[E[k, slot] - 1], mid)
    # element sizes are the step halved a whole number of times
    assert set(np.unique(sizes)) <= {step / 2 ** k for k in range(6)}
    # no element left mostly inside a hole
    assert not Q.mark_inside(c, E, mask).any()
    m.close()


def test_mesh_without_hole_is_the_uniform_mesh(aldic):
    coords, el = _uniform(384, 384, 16, 32, 16)
    mask = np.ones((384, 384))
    m = aldic.QuadtreeMesh.generate(coords, el, mask, 16)
    np.testing.assert_array_equal(m.coordinatesFEM, coords)
    np.testing.assert_array_equal(m.elementsFEM[:, :4], el)
    assert not m.elementsFEM[:, 4:].any()
    # only the border band (and two rings) is Dirichlet
    x = coords[m.dirichlet - 1, 0]
    y = coords[m.dirichlet - 1, 1]
    xmin, xmax, ymin, ymax = coords[:, 0].min(), coords[:, 0].max(), coords[:, 1].min(), coords[:, 1].max()
    edge = np.minimum.reduce([x - xmin, xmax - x, y - ymin, ymax - y])
    assert edge.max() <= 4 * 16


def test_mesh_rejects_fractional_coordinates(aldic):
    coords, el = _uniform(256, 256, 10, 20, 10)
    coords = coords + 0.5
    mask = _holes(256, 256, [(128, 128, 40)])
    with pytest.raises(aldic.AldicError):
        aldic.QuadtreeMesh.generate(coords, el, mask, 10)


def test_mesh_create_roundtrip(aldic):
    coords, el = _uniform(512, 512, 16, 32, 16)
    mask = _holes(512, 512, [(256, 256, 75)])
    c, E, d = Q.generate_quadtree_mesh(coords, el, mask, 16)
    m = aldic.QuadtreeMesh.create(c, E, d)
    np.testing.assert_array_equal(m.elementsFEM, E)
    np.testing.assert_array_equal(m.dirichlet, d)
    bad = E.copy()
    bad[0, 0] = 0
    with pytest.raises(aldic.AldicError):
        aldic.QuadtreeMesh.create(c, bad, d)
