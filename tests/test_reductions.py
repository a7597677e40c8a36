"""The transposed warp butterfly of k_icgn.cu (warp_sum_t) against per-value
butterflies (warp_sum), emulated over 32 lanes in FP64.

warp_sum: at each level o = 16, 8, 4, 2, 1 every lane adds its partner's
(lane ^ o) value to its own.  warp_sum_t: a lane holding m values keeps
the half its partner gives away (the upper half when lane & o, the lower
otherwise), adds the partner's copy of that half, and once it holds one
value continues as a plain butterfly.  The IC-GN setup (32 sums) and every
evaluation (8 sums; Subpb1: 4) rely on the two giving bit-identical totals,
with value i's total at lane i << (5 - log2 NV)."""
import numpy as np
import pytest


def butterfly(v):
    """v: (32,) one value per lane -> (32,) totals (identical in every lane)."""
    v = v.copy()
    for o in (16, 8, 4, 2, 1):
        v = v + v[np.arange(32) ^ o]
    return v


def transposed(vals):
    """vals: (32, NV) NV partial sums per lane -> (32,) v[0] of each lane."""
    nv = vals.shape[1]
    v = [vals[:, i].copy() for i in range(nv)]
    lanes = np.arange(32)
    for lvl in range(5):
        o = 16 >> lvl
        m = nv >> lvl
        partner = lanes ^ o
        if m > 1:
            hi = (lanes & o) != 0
            new = []
            for i in range(m // 2):
                lo_v, hi_v = v[i], v[i + m // 2]
                send = np.where(hi, lo_v, hi_v)
                keep = np.where(hi, hi_v, lo_v)
                new.append(keep + send[partner])
            v = new
        else:
            v[0] = v[0] + v[0][partner]
    return v[0]


@pytest.mark.parametrize("nv", [4, 8, 32])
def test_transposed_butterfly_bit_identical(nv):
    rng = np.random.default_rng(nv)
    # magnitudes spread over many binades, so that the order of the
    # additions shows in the rounding
    vals = rng.standard_normal((32, nv)) * np.exp(rng.uniform(-20, 20, (32, nv)))
    got = transposed(vals)
    shift = 5 - int(np.log2(nv))
    for i in range(nv):
        want = butterfly(vals[:, i])
        holders = np.arange(32)[(np.arange(32) >> shift) == i]
        assert np.array_equal(got[holders].view(np.int64), want[holders].view(np.int64)), i


def test_transposed_butterfly_differs_from_a_plain_sum():
    """Sanity: the test data are such that another summation order would
    round differently (so the bit-identity above is not vacuous)."""
    rng = np.random.default_rng(7)
    vals = rng.standard_normal(32) * np.exp(rng.uniform(-20, 20, 32))
    assert not np.array_equal(butterfly(vals)[0], np.add.reduce(vals[::-1]))
