"""The finite-difference Subproblem 2 on the GPU against the oracle: the
solve, the D2 strains and the whole FP64 frame with DICpara.Subpb2FDOrFEM = 1."""
import numpy as np
import pytest

from oracle import fd as FD

pytestmark = pytest.mark.gpu


def test_subpb2_fd_and_strain_match_oracle(aldic):
    rng = np.random.default_rng(4)
    M, N, h, mu = 37, 29, 8.0, 1e-3
    n = M * N
    U = rng.standard_normal(2 * n)
    F = 0.02 * rng.standard_normal(4 * n)
    ud = 0.002 * rng.standard_normal(4 * n)
    vd = 0.02 * rng.standard_normal(2 * n)
    for beta in (6.4e-5, 2.0e-2):
        ref = FD.subpb2_fd(M, N, h, beta, mu, U, F, ud, vd)
        out = aldic.subpb2_fd(M, N, h, beta, mu, U, F, ud, vd)
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-8)
    np.testing.assert_allclose(aldic.fd_strain(M, N, h, U), FD.fd_strain(M, N, h, U), atol=1e-13)


def test_frame_fd_fp64_matches_oracle(aldic, synth):
    wl = synth.workload("plain512")
    f, g = wl.images()
    ro = FD.frame_fd(f, g, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3)
    al = aldic.ALDIC(wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=3, precision=aldic.FP64,
                     subpb2="fd")
    al.set_images(f, g)
    r = al.frame()
    assert r["stats"]["beta"] == pytest.approx(ro["beta"], rel=1e-6)
    assert np.abs(r["U"] - ro["U"]).max() < 1e-4
    assert np.abs(r["F"] - ro["F"]).max() < 1e-4
    np.testing.assert_allclose(r["stats"]["update_y"], ro["update_y"], rtol=1e-3, atol=1e-7)
    ut, vt = synth.truth(wl, r["x0"], r["y0"])
    e = np.r_[r["U"][0::2] - ut, r["U"][1::2] - vt]
    assert np.sqrt(np.mean(e ** 2)) < 0.01
