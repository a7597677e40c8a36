"""aldic_b200 -- the AL-DIC hot path (integer search, IC-GN, ADMM Subproblems 1
and 2) as sm_100a CUDA kernels behind a C ABI (include/aldic_b200.h), with
this host package mirroring the reference MATLAB functions by name.

The package directory is ``2d_aldic_b200``; import it with
``importlib.import_module("2d_aldic_b200")``.
"""
from .api import (ALDIC, FP32, FP64, INIT_EXTRAP, INIT_GATED, INIT_GIVEN, INIT_PREV, INIT_SEARCH, INIT_ZERO,
                  INIT_SEARCH_MG,
                  ALDICSequence, Context, GenerateQuadtreeMesh, QuadtreeMesh, Subpb2Quadtree,
                  funGlobalNodalStrainQuadtree, quadtree_fill, ALDICQuadtree, icgn_flags,
                  quadtree_subset_sizes, InitNet, cnn_patches, cnn_to_init, subpb2_fd, fd_strain,
                  ComputeStrain, IntegerSearch, Init, LocalICGN, MeshSetUp, Subpb1,
                  Subpb2, ba_interp2, default_context, funGlobal_NodalStrainAvg, funICGN,
                  funICGN_Subpb1, funImgGradient, funIntegerSearch, funIntegerSearchMg, funNormalizeImg,
                  funSmoothDisp, funSmoothStrain, gridfit_springs, inpaint_nans, local_icgn)
from ._lib import AldicError, exported_symbols
from . import synth

__all__ = ["ALDIC", "ALDICSequence", "FP32", "FP64", "INIT_SEARCH", "INIT_PREV", "INIT_ZERO",
           "INIT_EXTRAP", "INIT_GIVEN", "INIT_SEARCH_MG", "INIT_GATED", "Context", "GenerateQuadtreeMesh", "QuadtreeMesh",
           "Subpb2Quadtree", "funGlobalNodalStrainQuadtree", "quadtree_fill", "ALDICQuadtree",
           "icgn_flags", "quadtree_subset_sizes", "InitNet", "cnn_patches", "cnn_to_init", "subpb2_fd", "fd_strain", "ComputeStrain", "IntegerSearch", "Init", "LocalICGN", "MeshSetUp",
           "Subpb1", "Subpb2", "ba_interp2", "default_context", "funGlobal_NodalStrainAvg",
           "funICGN", "funICGN_Subpb1", "funImgGradient", "funIntegerSearch", "funIntegerSearchMg", "funNormalizeImg",
           "funSmoothDisp", "funSmoothStrain", "gridfit_springs", "inpaint_nans", "local_icgn",
           "AldicError", "exported_symbols", "synth"]
