"""The 8-bit whole-field integer search against the oracle's per-point
funIntegerSearch restatement on larger grids: bit-identical u, v and
cc.max.  Steps that are multiples of 4 dividing the subset size run the
tiled kernel (every tile shape built: 16/4, 16/8, 24/8, 32/8, 32/16), step 10
the per-point kernel; grid rows of every length, a constant template patch
(normxcorr2 raises -> NaN) and a constant patch of the deformed image whose
maps hold dozens of exact ties."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,step,s", [(32, 8, 16), (32, 16, 24), (16, 8, 10), (32, 8, 5),
                                      (16, 4, 6), (24, 8, 12), (20, 10, 7)])
def test_segment_search_bit_exact(aldic, oracle, synth, w, step, s):
    W, H = 392, 328
    f = synth.speckle(W, H, 2500, 41)
    f[150:200, 100:170] = 77                 # constant templates inside
    g = synth.warp(f, lambda X, Y: (3.3 + 2.0 * np.sin(2 * np.pi * Y / 150),
                                    -2.1 + 1.5 * np.cos(2 * np.pi * X / 170)), 2.0, 41)
    _, mu_g, _ = oracle.normalize(g)
    x, y, u, v, cc = aldic.funIntegerSearch(f, g, s, [1, W], [1, H], w, step, 0, step,
                                            qfactors=False)
    xo, yo, uo, vo, cco, _ = oracle.int_search(f, g, mu_g, (1, W), (1, H), w, step, (s, s))
    assert u.shape == uo.shape
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_array_equal(y, yo)
    np.testing.assert_array_equal(np.isnan(u), np.isnan(uo))
    assert np.isnan(u).any()
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(v, vo)
    np.testing.assert_array_equal(cc["max"], cco)


def test_search_flat_deformed_patch(aldic, oracle, synth):
    """A constant region of g larger than the search windows: the interior
    entries of those maps are all 0 and each side of the outer ring holds
    cc - 2 = 33 identical values (the padded pixels read as the mean), so the
    maximum sits on the ring among dozens of exact ties, all of which the
    tiled kernel evaluates exactly (the first in map order wins)."""
    W, H = 300, 260
    f = synth.speckle(W, H, 1500, 43)
    g = synth.warp(f, lambda X, Y: (1.7 + 0 * X, -2.4 + 0 * Y), 2.0, 43)
    g[50:190, 70:230] = 77
    _, mu_g, _ = oracle.normalize(g)
    x, y, u, v, cc = aldic.funIntegerSearch(f, g, 16, [1, W], [1, H], 32, 8, 0, 8,
                                            qfactors=False)
    xo, yo, uo, vo, cco, _ = oracle.int_search(f, g, mu_g, (1, W), (1, H), 32, 8, (16, 16))
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(v, vo)
    np.testing.assert_array_equal(cc["max"], cco)
    ring = (np.abs(uo) == 17) | (np.abs(vo) == 17)   # integer peak on the ring
    assert ring.sum() > 5
