"""The GPU path against outputs the reference itself produced (loose pins; the
exact pins of the same fixtures run on the CPU in test_reference_pins.py):

* Sample12: ALDICQuadtree (main_ALDIC_Quadtree.m Sections 3-6) on the
  reference's images, ROI, mask and parameters reproduces the reference's
  quadtree mesh exactly and its ResultDisp{1}.U within the loose bounds of
  test_reference_pins.sample12_check, and the FP64 frame matches the oracle's
  restatement of the same frame within 1e-4 px;
* the manual's worked example: ALDIC with the FD Subproblem 2 and the
  reference's in-loop smoothing gives the printed ADMM update norms of steps
  2-5, and the FP64 frame matches the oracle's FD frame within 1e-4 px.
"""
import numpy as np
import pytest

from oracle import fd as FD
from oracle import quadtree as Q
from test_reference_pins import (MANUAL_SUBSETS, manual_check, manual_images, sample12,
                                 sample12_check)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def s12_oracle():
    z = sample12()
    return Q.frame(z["f"], z["g"], z["mask"].astype(np.float64), int(z["winsize"]),
                   int(z["winstepsize"]), int(z["search"][0]), tol=1e-2, gridx=tuple(z["gridx"]),
                   gridy=tuple(z["gridy"]))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sample12_quadtree_frame_matches_reference(aldic, s12_oracle, precision):
    z = sample12()
    qt = aldic.ALDICQuadtree(int(z["winsize"]), int(z["winstepsize"]), int(z["search"][0]), tol=1e-2,
                             precision=aldic.FP64 if precision == "fp64" else aldic.FP32,
                             gridx=tuple(z["gridx"]), gridy=tuple(z["gridy"]))
    qt.set_images(z["f"], z["g"], z["mask"].astype(np.float64))
    r = qt.frame()
    np.testing.assert_array_equal(r["coords"], z["coordinatesFEM"])
    np.testing.assert_array_equal(r["elems"], z["elementsFEM"])
    np.testing.assert_array_equal(r["dirichlet"], z["dirichlet"])
    sample12_check(r["U"], r["bad_icgn"], z, f"GPU {precision}")
    assert len(r["update_y"]) == int(z["ALSolveStep"]) - 1
    du = np.abs(r["U"] - s12_oracle["U"]).max()
    tol = 1e-4 if precision == "fp64" else 0.05
    assert du < tol, f"GPU {precision} vs oracle: {du:.3g} px"


@pytest.fixture(scope="module")
def manual_oracle():
    f, g, gx, gy = manual_images()
    return FD.frame_fd(f, g, 20, 10, 60, tol=1e-2, n_admm=4, gridx=gx, gridy=gy, smooth=True)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_manual_example_update_norms(aldic, manual_oracle, precision):
    f, g, gx, gy = manual_images()
    al = aldic.ALDIC(20, 10, 60, tol=1e-2, n_admm=4, smooth=True, subpb2="fd", gridx=gx, gridy=gy,
                     precision=aldic.FP64 if precision == "fp64" else aldic.FP32)
    al.set_images(f, g, roi=(gx[0], gx[1], gy[0], gy[1]))
    r = al.frame()
    assert r["M"] * r["N"] == MANUAL_SUBSETS
    st = r["stats"]
    assert st["bad_icgn"] == 0
    manual_check(st["update_y2"], st["update_y"], f"GPU {precision}")
    du = np.abs(r["U"] - manual_oracle["U"]).max()
    tol = 1e-4 if precision == "fp64" else 0.01
    assert du < tol, f"GPU {precision} vs oracle FD frame: {du:.3g} px"
