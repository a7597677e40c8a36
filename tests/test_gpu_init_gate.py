"""The gated external initial guess (ALDIC_INIT_GATED): a learned (or any
other) guess of U and the deformation gradient with a confidence per node;
nodes at or above the threshold start IC-GN from it, the others from the
integer search, which stays the fallback and the judge.

* nothing passes the gate -> the frame is bit-identical to the search frame;
* everything passes with the true field as the guess -> every node is taken
  and IC-GN converges from it to the search frame's result (within 0.01 px on
  99 % of the nodes).  The iteration count stays where it was (within 5 %):
  funICGN.m stops on the gradient norm relative to the start's own, so a
  start nearer the optimum takes as many Gauss-Newton steps to shrink its
  (smaller) norm by the same factor;
* a random confidence -> exactly the nodes at or above the threshold."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(aldic, synth):
    wl = synth.workload("plain512")
    f, g = wl.images()
    al = aldic.ALDIC(wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=2, precision=aldic.FP32)
    al.set_images(f, g)
    r = al.frame()
    return wl, al, r


def test_gate_closed_is_the_search_frame(aldic, setup):
    wl, al, r = setup
    n = r["M"] * r["N"]
    al.set_init_gated(np.zeros(2 * n), np.zeros(4 * n), np.zeros(n, np.float32), 0.5)
    rg = al.frame(init=aldic.INIT_GATED)
    assert rg["stats"]["gated_init"] == 0
    for k in ("U", "F", "iters", "x0", "y0"):
        np.testing.assert_array_equal(rg[k], r[k])


def test_gate_open_with_true_field(aldic, synth, setup):
    wl, al, r = setup
    n = r["M"] * r["N"]
    ut, vt = synth.truth(wl, r["x0"], r["y0"])
    U0 = np.empty(2 * n)
    U0[0::2], U0[1::2] = ut, vt
    # the workload's affine field: u = 0.5 + 0.01 x, v = -0.3 + 0.005 y
    F0 = np.zeros(4 * n)
    F0[0::4], F0[3::4] = 0.01, 0.005
    al.set_init_gated(U0, F0, np.ones(n, np.float32), 0.5)
    rg = al.frame(init=aldic.INIT_GATED)
    st, s0 = rg["stats"], r["stats"]
    assert st["gated_init"] == n
    d = np.abs(rg["U"] - r["U"]).reshape(-1, 2).max(1)
    assert np.mean(d < 0.01) >= 0.99, np.mean(d < 0.01)
    assert st["mean_iters_icgn"] <= 1.05 * s0["mean_iters_icgn"]
    print(f"mean IC-GN iterations: search start {s0['mean_iters_icgn']:.3f}, "
          f"true-field start {st['mean_iters_icgn']:.3f}")


def test_gate_threshold(aldic, setup):
    wl, al, r = setup
    n = r["M"] * r["N"]
    conf = np.random.default_rng(1).random(n).astype(np.float32)
    U0 = np.empty(2 * n)
    U0[0::2], U0[1::2] = 0.5, -0.3
    al.set_init_gated(U0, None, conf, 0.7)
    rg = al.frame(init=aldic.INIT_GATED)
    assert rg["stats"]["gated_init"] == int((conf >= 0.7).sum())
