"""Image sequences on the GPU against the oracle: every initial-guess mode of
main_ALDIC.m's frame loop (search, reference update with U0 = 0, previous U,
extrapolation, caller-given U0) on a 16-bit sequence."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def seq16(synth):
    # 512^2 uint16, 8 frames: 0.2 %/frame stretch, 0.5 px sinusoid, noise 30
    sq = synth.sequence("sequence4096", scale_down=8, n_frames=8)
    frames = sq.frames()
    return sq, frames, [f.numpy() for f in frames]


def test_sequence_fp64_matches_oracle(aldic, oracle, seq16):
    import torch
    sq, frames, np_frames = seq16
    kw = dict(winsize=sq.winsize, step=sq.step, search=sq.search, tol=sq.tol, n_admm=2)
    seq = aldic.ALDICSequence(inc_unit=3, n_search=2, precision=aldic.FP64, **kw)
    res = list(seq.run([f.cuda() for f in frames]))
    modes = [r["init"] for r in res]
    assert modes == [aldic.INIT_SEARCH, aldic.INIT_SEARCH, aldic.INIT_EXTRAP, aldic.INIT_ZERO,
                     aldic.INIT_PREV, aldic.INIT_EXTRAP, aldic.INIT_ZERO]
    hist = []
    for r in res:
        s, mode, ref = r["img_seq_num"], r["init"], r["ref_index"]
        U0 = {aldic.INIT_SEARCH: None,
              aldic.INIT_ZERO: lambda: np.zeros_like(hist[-1]),
              aldic.INIT_PREV: lambda: hist[-1],
              aldic.INIT_EXTRAP: lambda: 2 * hist[-1] - hist[-2]}[mode]
        ro = oracle.frame(np_frames[ref], np_frames[s - 1], sq.winsize, sq.step, sq.search,
                          tol=sq.tol, n_admm=2, U0=U0() if U0 else None)
        hist.append(ro["U"])
        U = r["U"].cpu().numpy()
        np.testing.assert_array_equal(r["x0"].cpu().numpy(), ro["x0"])
        assert np.abs(U - ro["U"]).max() < 1e-4, (s, mode)
        ut, vt = sq.truth(s - 1, ref, ro["x0"], ro["y0"])
        e = np.r_[U[0::2] - ut, U[1::2] - vt]
        assert np.sqrt(np.mean(e ** 2)) < 0.02, (s, mode)
        assert r["latency_ms"] > 0
    torch.cuda.synchronize()


def test_given_init_equals_previous(aldic, seq16):
    sq, frames, _ = seq16
    ctx = aldic.Context(0)
    al = aldic.ALDIC(sq.winsize, sq.step, sq.search, tol=sq.tol, n_admm=1, precision=aldic.FP32,
                     ctx=ctx)
    al.set_images(frames[0].cuda(), frames[1].cuda())
    with pytest.raises(aldic.AldicError):
        al.frame(init=aldic.INIT_PREV)          # no previous frame yet
    r0 = al.frame()                              # integer search
    al.set_images(g=frames[2].cuda())
    r1 = al.frame(init=aldic.INIT_PREV)
    al.set_init(r0["U"])
    r2 = al.frame(init=aldic.INIT_GIVEN)
    for k in ("U", "F", "iters"):
        np.testing.assert_array_equal(r1[k], r2[k])
    r3 = al.frame(init=aldic.INIT_EXTRAP)        # U0 = 2 U(r2) - U(r1) = U(r1)
    al.set_init(r1["U"])
    r4 = al.frame(init=aldic.INIT_GIVEN)
    np.testing.assert_array_equal(r3["U"], r4["U"])
    ctx.close()
