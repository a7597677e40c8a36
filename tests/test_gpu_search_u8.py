"""The 8-bit whole-field integer search against the oracle's per-point
funIntegerSearch restatement on larger grids: bit-identical u, v and
cc.max for subsets of 32 and 16 px, steps 8 and 16, search radii 5 to 24,
grid rows of every length and a constant patch (normxcorr2 raises -> NaN)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,step,s", [(32, 8, 16), (32, 16, 24), (16, 8, 10), (32, 8, 5)])
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
