"""Writes the reference-held fixtures of the parity pins (test infrastructure).

    python tests/golden/make_reference_fixtures.py <path of the 2D_ALDIC checkout>
    (or ALDIC_REFERENCE=<path> python tests/golden/make_reference_fixtures.py)

sample12.npz -- the reference's own quadtree run on its Sample12 images:
  * Images_Quadtree_demo/Images_Sample12/oht_cfrp_00.tiff, oht_cfrp_11.tiff
    (400 x 1040, 8-bit palette images with an identity grey palette, so the
    palette indices are the grey levels MATLAB's imread returns);
  * results_ForQuadtree_Sample12/results_oht_cfrp_11_ws32_st16.mat: DICpara
    (winsize 32, winstepsize 16, gridxyROIRange x 40..354 / y 14..1026,
    ImgRefMask, SizeOfFFTSearchRegion 13, elementMinSize 2), the quadtree
    mesh GenerateQuadtreeMesh.m produced (coordinatesFEM, elementsFEM,
    dirichlet = markCoordHoleEdge), the uniform search grid x0/y0, the frame's
    result ResultDisp{1}.U / ResultDefGrad{1}.F and ALSub1BadPtNum.
  Arrays are stored in C order with images and the mask as (H, W) = (y, x).

frac_heter_manual.npz -- the images of the reference manual's worked example
  (manual_v4.2 section 12: img_0000.tif / img_0570.tif, 822 x 1242 16-bit),
  cropped to columns 200..822 (1-based; the ROI 310..760 x 70..1146 with the
  60 px search and the 20 px subsets stays > 100 px inside the crop, so the
  search grid, normalisation and every subset read are those of the full
  image), with the crop's column offset.  The manual's printed ADMM update
  norms are constants in the tests that use this fixture.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CROP_X0 = 199          # 0-based first column kept of the manual images


def _img(path):
    from PIL import Image
    im = Image.open(path)
    if im.mode == "P":
        pal = np.asarray(im.getpalette(), np.int64).reshape(-1, 3)
        if not (np.array_equal(pal[:, 0], np.arange(len(pal)))
                and np.array_equal(pal[:, 0], pal[:, 1]) and np.array_equal(pal[:, 1], pal[:, 2])):
            raise ValueError(f"{path}: palette is not the identity grey ramp")
    return np.asarray(im)


def sample12(ref):
    import scipy.io as sio
    m = sio.loadmat(os.path.join(ref, "results_ForQuadtree_Sample12", "results_oht_cfrp_11_ws32_st16.mat"),
                    squeeze_me=True, struct_as_record=False)
    dm, dp = m["DICmesh"], m["DICpara"]
    d = os.path.join(ref, "Images_Quadtree_demo", "Images_Sample12")
    f = _img(os.path.join(d, "oht_cfrp_00.tiff"))
    g = _img(os.path.join(d, "oht_cfrp_11.tiff"))
    mask = np.ascontiguousarray(np.asarray(dp.ImgRefMask).T.astype(np.uint8))   # Img(x,y) -> (H, W)
    assert f.shape == g.shape == mask.shape
    gr = dp.gridxyROIRange
    np.savez_compressed(
        os.path.join(HERE, "sample12.npz"),
        f=f, g=g, mask=mask,
        gridx=np.asarray(gr.gridx, np.int32), gridy=np.asarray(gr.gridy, np.int32),
        winsize=np.int32(dp.winsize), winstepsize=np.int32(dp.winstepsize),
        search=np.asarray(dp.SizeOfFFTSearchRegion, np.int32), elementMinSize=np.int32(dm.elementMinSize),
        x0=np.asarray(dm.x0, np.float64).T.copy(), y0=np.asarray(dm.y0, np.float64).T.copy(),  # (N, M)
        coordinatesFEM=np.asarray(dm.coordinatesFEM, np.float64),
        elementsFEM=np.asarray(dm.elementsFEM, np.int64),
        dirichlet=np.asarray(dm.dirichlet, np.int64),
        markCoordHoleEdge=np.asarray(dm.markCoordHoleEdge, np.int64),
        U=np.asarray(m["ResultDisp"].U, np.float64),
        F=np.asarray(m["ResultDefGrad"].F, np.float64),
        ALSub1BadPtNum=np.asarray(m["ResultDisp"].ALSub1BadPtNum, np.int64),
        ALSolveStep=np.int32(m["ALSolveStep"]))


def frac_heter(ref):
    f = _img(os.path.join(ref, "img_0000.tif"))
    g = _img(os.path.join(ref, "img_0570.tif"))
    assert f.dtype == np.uint16 and f.shape == (1242, 822)
    np.savez_compressed(os.path.join(HERE, "frac_heter_manual.npz"),
                        f=np.ascontiguousarray(f[:, CROP_X0:]), g=np.ascontiguousarray(g[:, CROP_X0:]),
                        crop_x0=np.int32(CROP_X0))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ALDIC_REFERENCE")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: make_reference_fixtures.py <2D_ALDIC checkout> (or set ALDIC_REFERENCE)")
    sample12(ref)
    frac_heter(ref)


if __name__ == "__main__":
    main()
