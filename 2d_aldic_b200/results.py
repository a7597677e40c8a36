"""Results files in the reference's layout (main_ALDIC.m:469-473): a MATLAB
.mat file named results_<image>_ws<winsize>_st<winstepsize>.mat holding
file_name, DICpara, DICmesh, ResultDisp, ResultDefGrad, ResultFEMesh,
ResultFEMeshEachFrame, ALSub1Time, ALSub2Time and ALSolveStep, with the
per-frame cells as structs (ResultDisp{k}.U, ResultDefGrad{k}.F).  Host-side
bookkeeping: the arrays come from the library's frames."""
from __future__ import annotations

import os

import numpy as np


def results_name(file_name, DICpara) -> str:
    """main_ALDIC.m:470-471: results_<last image name>_ws<winsize>_st<winstepsize>.mat."""
    last = file_name[-1] if isinstance(file_name, (list, tuple)) else file_name
    img = os.path.splitext(os.path.basename(str(last)))[0]
    ws = int(np.mean(DICpara["winsize"]))
    st = int(np.mean(DICpara["winstepsize"]))
    return f"results_{img}_ws{ws}_st{st}.mat"


def _cell(items):
    c = np.empty((len(items), 1), dtype=object)
    for k, v in enumerate(items):
        c[k, 0] = v
    return c


def _col(a):
    return np.asarray(a, np.float64).reshape(-1, 1)


def save_results(path, file_name, DICpara, DICmesh, frames, ALSub1Time=None, ALSub2Time=None,
                 ALSolveStep=None):
    """Write the reference's results file.  frames: one dict per deformed
    image with U (2n), F (4n) and optionally ALSub1BadPtNum, coordinatesFEM,
    elementsFEM (the mesh of that frame; default DICmesh's)."""
    import scipy.io
    disp, grad, mesh_each = [], [], []
    for fr in frames:
        d = {"U": _col(fr["U"])}
        if "ALSub1BadPtNum" in fr:
            d["ALSub1BadPtNum"] = _col(fr["ALSub1BadPtNum"])
        disp.append(d)
        grad.append({"F": _col(fr["F"])})
        mesh_each.append({"coordinatesFEM": np.asarray(fr.get("coordinatesFEM", DICmesh["coordinatesFEM"]), np.float64),
                          "elementsFEM": np.asarray(fr.get("elementsFEM", DICmesh["elementsFEM"]), np.float64)})
    mesh = {k: (np.asarray(v, np.float64) if not isinstance(v, (str, dict)) else v)
            for k, v in DICmesh.items() if v is not None and not (isinstance(v, list) and len(v) == 0)}
    first = {"coordinatesFEM": mesh["coordinatesFEM"], "elementsFEM": mesh["elementsFEM"],
             "winsize": float(np.mean(DICpara["winsize"])),
             "winstepsize": float(np.mean(DICpara["winstepsize"]))}
    out = {
        "file_name": _cell([str(f) for f in (file_name if isinstance(file_name, (list, tuple)) else [file_name])]),
        "DICpara": {k: v for k, v in DICpara.items() if v is not None},
        "DICmesh": mesh,
        "ResultDisp": _cell(disp),
        "ResultDefGrad": _cell(grad),
        "ResultFEMesh": _cell([first]),
        "ResultFEMeshEachFrame": _cell(mesh_each),
        "ALSub1Time": _col(ALSub1Time if ALSub1Time is not None else np.zeros(6)),
        "ALSub2Time": _col(ALSub2Time if ALSub2Time is not None else np.zeros(6)),
        "ALSolveStep": float(ALSolveStep if ALSolveStep is not None else 0),
    }
    scipy.io.savemat(path, out, do_compression=True)
    return path


def load_results(path):
    """Read a results file written by save_results (or by the reference):
    dict with file_name, DICpara, DICmesh and frames (U, F per frame)."""
    import scipy.io
    m = scipy.io.loadmat(path, squeeze_me=True, struct_as_record=False)
    disp = np.atleast_1d(m["ResultDisp"])
    grad = np.atleast_1d(m["ResultDefGrad"])
    frames = [{"U": np.asarray(d.U, np.float64).reshape(-1), "F": np.asarray(g.F, np.float64).reshape(-1)}
              for d, g in zip(disp, grad)]
    return {"file_name": list(np.atleast_1d(m["file_name"])), "DICpara": m["DICpara"],
            "DICmesh": m["DICmesh"], "frames": frames}
