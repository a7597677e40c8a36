"""Results files (main_ALDIC.m:469-473) and the strain post-processing
oracle (ComputeStrain.m).  CPU only."""
import importlib

import numpy as np

from oracle import strain as S


def test_results_file_roundtrip(tmp_path):
    R = importlib.import_module("2d_aldic_b200.results")
    rng = np.random.default_rng(0)
    M, N = 5, 4
    coords = np.stack(np.meshgrid(np.arange(M) * 8.0 + 20, np.arange(N) * 8.0 + 20), -1).reshape(-1, 2)
    mesh = {"coordinatesFEM": coords, "elementsFEM": np.array([[1, 2, 7, 6]]), "M": M, "N": N}
    para = {"winsize": 16, "winstepsize": 8, "ImgSeqIncUnit": 11}
    frames = [{"U": rng.standard_normal(2 * M * N), "F": rng.standard_normal(4 * M * N),
               "ALSub1BadPtNum": np.arange(6.0)} for _ in range(3)]
    name = R.results_name(["a/img_0001.tif", "a/img_0570.tif"], para)
    assert name == "results_img_0570_ws16_st8.mat"
    p = R.save_results(str(tmp_path / name), ["img_0001.tif", "img_0570.tif"], para, mesh, frames,
                       ALSolveStep=4)
    back = R.load_results(p)
    assert back["file_name"] == ["img_0001.tif", "img_0570.tif"]
    for a, b in zip(frames, back["frames"]):
        np.testing.assert_array_equal(a["U"], b["U"])
        np.testing.assert_array_equal(a["F"], b["F"])
    assert int(back["DICpara"].winstepsize) == 8
    np.testing.assert_array_equal(back["DICmesh"].coordinatesFEM, coords)


def test_strain_oracle_affine_exact():
    M, N, h = 9, 7, 8.0
    k = np.arange(M * N)
    x, y = h * (k % M), h * (k // M)
    U = np.empty(2 * M * N)
    U[0::2] = 0.5 + 0.01 * x - 0.004 * y
    U[1::2] = -1.0 + 0.002 * x + 0.03 * y
    g = np.array([0.01, 0.002, -0.004, 0.03])
    for method, rad in ((1, 1), (2, 2), (3, 1)):
        fs, ff = S.compute_strain(M, N, h, method, rad, 0, U)
        # method 3 keeps funGlobal_NodalStrainAvg's slot order [du/dx du/dy dv/dx dv/dy]
        want = g[[0, 2, 1, 3]] if method == 3 else g
        np.testing.assert_allclose(fs.reshape(-1, 4), np.tile(want, (M * N, 1)), atol=1e-13)
    _, ff = S.compute_strain(M, N, h, 1, 1, 2, U)
    ux, vx, uy, vy = g
    np.testing.assert_allclose(ff.reshape(-1, 4)[0], [0.5 * (2 * ux - ux ** 2 - vx ** 2),
                                                     0.5 * (vx + uy - uy * ux - vy * vx),
                                                     0.5 * (uy + vx - ux * uy - vx * vy),
                                                     0.5 * (2 * vy - uy ** 2 - vy ** 2)], atol=1e-15)
