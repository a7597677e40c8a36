"""Image sequences (main_ALDIC.m:53-147): the frame loop's choice of initial
guess and reference image, and the oracle's later-frame path.  CPU only."""
import numpy as np
import pytest


def test_sequence_plan_follows_main_aldic(aldic):
    seq = aldic.ALDICSequence.__new__(aldic.ALDICSequence)
    seq.inc_unit, seq.n_search, seq.predictor = 10, 5, "extrap"
    plan = seq.plan(50)
    assert [p[0] for p in plan] == list(range(2, 51))
    modes = {s: m for s, m, _, _ in plan}
    refs = {s: r for s, _, r, _ in plan}
    upd = [s for s, _, _, u in plan if u]
    # ImgSeqNum < 7: integer search against the first image
    assert all(modes[s] == aldic.INIT_SEARCH for s in range(2, 7))
    # reference update when mod(ImgSeqNum - 2, 10) == 0 (and no search that frame):
    # the previous image becomes the reference, U0 = 0
    assert upd == [12, 22, 32, 42]
    assert all(modes[s] == aldic.INIT_ZERO and refs[s] == s - 2 for s in upd)
    assert all(refs[s] == 0 for s in range(2, 12)) and refs[21] == 10 and refs[50] == 40
    # first frame after an update: the previous U; later: extrapolation
    assert all(modes[s + 1] == aldic.INIT_PREV and modes[s + 2] == aldic.INIT_EXTRAP for s in upd)
    assert modes[7] == aldic.INIT_EXTRAP
    # accumulative mode never changes the reference
    seq.inc_unit = None
    assert not any(u for *_, u in seq.plan(50))
    seq.predictor = "previous"
    assert {m for _, m, _, _ in seq.plan(12)} == {aldic.INIT_SEARCH, aldic.INIT_PREV}


def test_oracle_given_U0_equals_search_path(oracle, synth):
    """orc_frame with init_U = the U0 that its own search + Init produce gives
    the identical frame: the later-frame path differs only in where U0 comes
    from."""
    wl = synth.workload("plain512", scale_down=2)
    f, g = wl.images()
    H, W = f.shape
    kw = dict(tol=wl.tol, n_admm=2)
    ro = oracle.frame(f, g, wl.winsize, wl.step, wl.search, **kw)
    _, mg, _ = oracle.normalize(g)
    s2 = (wl.search, wl.search)
    x, y, u, v, cc, _ = oracle.int_search(f, g, mg, (1, W), (1, H), wl.winsize, wl.step, s2)
    M, N = ro["M"], ro["N"]
    assert u.shape == (N, M)
    np.testing.assert_array_equal(x.reshape(-1), ro["x0"])
    ug = oracle.inpaint_springs(M, N, u.reshape(-1))
    vg = oracle.inpaint_springs(M, N, v.reshape(-1))
    U0 = np.empty(2 * M * N)
    U0[0::2], U0[1::2] = ug, vg
    rg = oracle.frame(f, g, wl.winsize, wl.step, wl.search, U0=U0, **kw)
    np.testing.assert_array_equal(rg["x0"], ro["x0"])
    np.testing.assert_array_equal(rg["y0"], ro["y0"])
    for k in ("U", "F", "iters_icgn"):
        np.testing.assert_array_equal(rg[k], ro[k])


def test_sequence_truth_composes(synth):
    """truth(k, r) is the displacement between the configurations of frames r
    and k: going r -> k equals going 0 -> k minus 0 -> r at the same material
    point."""
    sq = synth.sequence("sequence4096", scale_down=8, n_frames=6)
    x = np.array([60.0, 250.0, 400.0])
    y = np.array([90.0, 256.0, 430.0])
    ur, vr = sq.truth(3, 0, x, y)                       # 0 -> 3 at X
    u5, v5 = sq.truth(5, 0, x, y)                       # 0 -> 5 at X
    uk, vk = sq.truth(5, 3, x + ur, y + vr)             # 3 -> 5 at x3 = X + u3
    np.testing.assert_allclose(uk, u5 - ur, atol=1e-8)
    np.testing.assert_allclose(vk, v5 - vr, atol=1e-8)
    with pytest.raises(ValueError):
        from importlib import import_module
        import_module("2d_aldic_b200").ALDICSequence(predictor="pod")
