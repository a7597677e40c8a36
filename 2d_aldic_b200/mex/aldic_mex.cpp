// aldic_mex.cpp -- MEX gateway for the batched hot path (one call per frame
// instead of one funICGN / funICGN_Subpb1 call per subset).
//
//     mex -R2018a aldic_mex.cpp -I<repo>/include -L<repo>/2d_aldic_b200 -laldic_b200
//
// Commands (the first argument), mirroring the reference's functions:
//   [U,F,ConvItPerEle,HtempPar] = aldic_mex('icgn', U0, coordinatesFEM, DfDx, DfDy,
//                                           ImgRef, ImgDef, winsize, tol)
//       the per-node loop of LocalICGN.m:64-81 (funICGN.m for every node)
//   [U,ConvItPerEle] = aldic_mex('subpb1', UOld, FOld, vdual, coordinatesFEM, DfDx,
//                                DfDy, ImgRef, ImgDef, HtempPar, winsize, mu, tol)
//       the per-node loop of Subpb1.m:64-103 (funICGN_Subpb1.m for every node)
//   Uhat = aldic_mex('subpb2', M, N, winstepsize, beta, mu, U, F, udual, vdual)
//       Subpb2.m on the uniform mesh of MeshSetUp.m
//   F = aldic_mex('strain', M, N, winstepsize, U)
//       funGlobal_NodalStrainAvg.m on the uniform mesh
//   [x0,y0,u,v,ccmax] = aldic_mex('searchmg', ImgRef, ImgDef, gridx, gridy, winsize,
//                                 winstepsize)
//       funIntegerSearchMg.m (IntegerSearch.m:117-120), ny x nx outputs
//   [FStrain,FStrainFinite] = aldic_mex('computestrain', M, N, winstepsize, method, rad,
//                                       straintype, U, F)
//       ComputeStrain.m Section 8 (F is read by method 0 only; pass [] otherwise)
//   [x,y,u,v,ccmax,qfactors] = aldic_mex('intsearch', f, g, tempSizeOfSearchRegion, gridx,
//                                        gridy, winsize, winstepsize)
//       funIntegerSearch.m:3 whole field (the call of IntegerSearch.m:54 with
//       tempNoOfInitPt = 0): x, y, u, v, ccmax are ny x nx, qfactors n x 2
//       (cc.max and cc.qfactors of the reference's cc struct).  f, g: W x H
//       double (normalised, as IntegerSearch passes them) or uint8/uint16 raw
//       images (exact integer correlation, statistics over gridx x gridy)
//   Uhat = aldic_mex('subpb2qt', coordinatesFEM, elementsFEM, dirichlet, beta, mu, U, F)
//       Subpb2Quadtree.m:1 (GaussPtOrder 2, alpha 0) on a DICmesh of the
//       quadtree path: coordinatesFEM n x 2, elementsFEM ne x 8 (hanging nodes
//       in columns 5-8, 0 = none), dirichlet the node list
//   [x0,y0,U,F,ConvItPerEle,stats] = aldic_mex('frame', ImgRef, ImgDef, winsize,
//        winstepsize, tempSizeOfSearchRegion, gridx, gridy, tol, nADMM, Subpb2FDOrFEM,
//        smooth)
//       one frame of main_ALDIC.m Sections 3-6 (whole-field search, LocalICGN,
//       beta sweep, nADMM ADMM steps; Subpb2FDOrFEM 1 = FD, 2 = FE; smooth 1 =
//       the funSmoothDisp/funSmoothStrain calls): x0, y0 M x N, U 2MN, F 4MN,
//       ConvItPerEle MN x 1; stats = [beta, LocalICGNBadPtNum, UpdateY of each
//       ADMM step] (all nADMM steps run: compare UpdateY with tol2 = 1e-4 of
//       main_ALDIC.m:354 to see where the reference would have stopped).
//       ImgRef/ImgDef raw uint8/uint16 or double W x H
// ImgRef/ImgDef are the normalised W x H doubles; DfDx/DfDy are the reference's
// (W-6) x (H-6) Df.DfDx/Df.DfDy.  The GPU context persists across calls
// (mexLock), images and gradients are re-uploaded on every icgn/subpb1 call.
#include <mex.h>

#include <cstring>
#include <string>
#include <vector>

#include "aldic_b200.h"

static aldic_ctx *g_ctx = nullptr;

static void release() {
  if (g_ctx) aldic_ctx_destroy(g_ctx);
  g_ctx = nullptr;
}

static void check(int rc) {
  if (rc != ALDIC_OK) mexErrMsgIdAndTxt("aldic:call", "%s", aldic_last_error());
}

static aldic_ctx *ctx() {
  if (!g_ctx) {
    check(aldic_ctx_create(0, &g_ctx));
    mexLock();
    mexAtExit(release);
  }
  return g_ctx;
}

static const double *dbl(const mxArray *a, const char *what) {
  if (!mxIsDouble(a)) mexErrMsgIdAndTxt("aldic:type", "%s must be double", what);
  return (const double *)mxGetData(a);
}

// Df.DfDx is (W-6) x (H-6); the library wants W x H with a zero 3-pixel border
static std::vector<double> expand_df(const mxArray *d, size_t W, size_t H) {
  if (mxGetM(d) != W - 6 || mxGetN(d) != H - 6)
    mexErrMsgIdAndTxt("aldic:size", "Df.DfDx/DfDy must be (W-6) x (H-6)");
  std::vector<double> out(W * H, 0.0);
  const double *s = dbl(d, "Df");
  for (size_t y = 0; y < H - 6; ++y)
    std::memcpy(&out[(y + 3) * W + 3], s + y * (W - 6), sizeof(double) * (W - 6));
  return out;
}

// uint8 / uint16 / double image class -> library dtype
static int img_dtype(const mxArray *a, const char *what) {
  if (mxIsUint8(a)) return ALDIC_U8;
  if (mxIsUint16(a)) return ALDIC_U16;
  if (mxIsDouble(a)) return ALDIC_F64;
  mexErrMsgIdAndTxt("aldic:type", "%s must be uint8, uint16 or double", what);
  return -1;
}

static void pair2(const mxArray *a, const char *what, int out[2]) {
  if (!mxIsDouble(a) || mxGetNumberOfElements(a) < 1 || mxGetNumberOfElements(a) > 2)
    mexErrMsgIdAndTxt("aldic:size", "%s is a double scalar or [a b]", what);
  const double *d = (const double *)mxGetData(a);
  out[0] = (int)d[0];
  out[1] = (int)d[mxGetNumberOfElements(a) - 1];
}

// hand the first max(nlhs, 1) of k arrays to MATLAB and free the rest
// (plhs has room for max(nlhs, 1) entries only)
static void give_outputs(mxArray **o, int k, int nlhs, mxArray *plhs[]) {
  const int keep = nlhs > 1 ? nlhs : 1;
  for (int i = 0; i < k; ++i) {
    if (i < keep) plhs[i] = o[i];
    else mxDestroyArray(o[i]);
  }
}

static void load_fields(const mxArray *DfDx, const mxArray *DfDy, const mxArray *f,
                        const mxArray *g) {
  const size_t W = mxGetM(f), H = mxGetN(f);
  if (mxGetM(g) != W || mxGetN(g) != H) mexErrMsgIdAndTxt("aldic:size", "ImgRef/ImgDef differ");
  std::vector<double> gx = expand_df(DfDx, W, H), gy = expand_df(DfDy, W, H);
  check(aldic_set_fields(ctx(), dbl(f, "ImgRef"), dbl(g, "ImgDef"), gx.data(), gy.data(), (int)W,
                         (int)H));
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  if (nrhs < 1 || mxGetClassID(prhs[0]) != mxCHAR_CLASS)
    mexErrMsgIdAndTxt("aldic:usage", "aldic_mex(command, ...)");
  char cmd[32] = {0};
  const unsigned short *cs = (const unsigned short *)mxGetData(prhs[0]);
  for (size_t i = 0; i < mxGetNumberOfElements(prhs[0]) && i < 31; ++i) cmd[i] = (char)cs[i];
  const std::string c(cmd);
  if (c == "icgn") {
    if (nrhs != 9) mexErrMsgIdAndTxt("aldic:usage", "icgn takes 8 arguments");
    load_fields(prhs[3], prhs[4], prhs[5], prhs[6]);
    const size_t n = mxGetM(prhs[2]);
    if (mxGetN(prhs[2]) != 2 || mxGetNumberOfElements(prhs[1]) != 2 * n)
      mexErrMsgIdAndTxt("aldic:size", "coordinatesFEM is n x 2 and U0 is 2n");
    plhs[0] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
    plhs[1] = mxCreateDoubleMatrix(4 * n, 1, mxREAL);
    mwSize d1[2] = {n, 1};
    mxArray *it = mxCreateNumericArray(2, d1, mxINT32_CLASS, mxREAL);
    mxArray *H21 = mxCreateDoubleMatrix(n, 21, mxREAL);
    check(aldic_icgn(ctx(), dbl(prhs[2], "coordinatesFEM"), (int64_t)n, dbl(prhs[1], "U0"),
                     nullptr, (int)mxGetScalar(prhs[7]), mxGetScalar(prhs[8]), ALDIC_FP64,
                     mxGetPr(plhs[0]), mxGetPr(plhs[1]), (int32_t *)mxGetData(it),
                     mxGetPr(H21)));
    if (nlhs > 2) plhs[2] = it; else mxDestroyArray(it);
    if (nlhs > 3) plhs[3] = H21; else mxDestroyArray(H21);
  } else if (c == "subpb1") {
    if (nrhs != 13) mexErrMsgIdAndTxt("aldic:usage", "subpb1 takes 12 arguments");
    load_fields(prhs[5], prhs[6], prhs[7], prhs[8]);
    const size_t n = mxGetM(prhs[4]);
    plhs[0] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
    mwSize d1[2] = {n, 1};
    mxArray *it = mxCreateNumericArray(2, d1, mxINT32_CLASS, mxREAL);
    check(aldic_subpb1(ctx(), dbl(prhs[4], "coordinatesFEM"), (int64_t)n, dbl(prhs[1], "UOld"),
                       dbl(prhs[2], "FOld"), dbl(prhs[3], "vdual"), dbl(prhs[9], "HtempPar"),
                       nullptr, (int)mxGetScalar(prhs[10]), mxGetScalar(prhs[11]),
                       mxGetScalar(prhs[12]), ALDIC_FP64, mxGetPr(plhs[0]),
                       (int32_t *)mxGetData(it)));
    if (nlhs > 1) plhs[1] = it; else mxDestroyArray(it);
  } else if (c == "subpb2") {
    if (nrhs != 10) mexErrMsgIdAndTxt("aldic:usage", "subpb2 takes 9 arguments");
    const int M = (int)mxGetScalar(prhs[1]), N = (int)mxGetScalar(prhs[2]);
    plhs[0] = mxCreateDoubleMatrix(2 * (size_t)M * N, 1, mxREAL);
    check(aldic_subpb2(ctx(), M, N, mxGetScalar(prhs[3]), mxGetScalar(prhs[4]),
                       mxGetScalar(prhs[5]), dbl(prhs[6], "U"), dbl(prhs[7], "F"),
                       dbl(prhs[8], "udual"), dbl(prhs[9], "vdual"), mxGetPr(plhs[0])));
  } else if (c == "strain") {
    if (nrhs != 5) mexErrMsgIdAndTxt("aldic:usage", "strain takes 4 arguments");
    const int M = (int)mxGetScalar(prhs[1]), N = (int)mxGetScalar(prhs[2]);
    plhs[0] = mxCreateDoubleMatrix(4 * (size_t)M * N, 1, mxREAL);
    check(aldic_nodal_strain(ctx(), M, N, mxGetScalar(prhs[3]), dbl(prhs[4], "U"),
                             mxGetPr(plhs[0])));
  } else if (c == "searchmg") {
    if (nrhs != 7) mexErrMsgIdAndTxt("aldic:usage", "searchmg takes 6 arguments");
    const size_t W = mxGetM(prhs[1]), H = mxGetN(prhs[1]);
    if (mxGetM(prhs[2]) != W || mxGetN(prhs[2]) != H)
      mexErrMsgIdAndTxt("aldic:size", "ImgRef/ImgDef differ");
    if (mxGetNumberOfElements(prhs[3]) != 2 || mxGetNumberOfElements(prhs[4]) != 2)
      mexErrMsgIdAndTxt("aldic:size", "gridx and gridy are [first last]");
    std::vector<double> zeros(W * H, 0.0);  // gradients: not used by the search
    check(aldic_set_fields(ctx(), dbl(prhs[1], "ImgRef"), dbl(prhs[2], "ImgDef"), zeros.data(),
                           zeros.data(), (int)W, (int)H));
    const double *gxd = dbl(prhs[3], "gridx"), *gyd = dbl(prhs[4], "gridy");
    const int gx[2] = {(int)gxd[0], (int)gxd[1]}, gy[2] = {(int)gyd[0], (int)gyd[1]};
    const int step = (int)mxGetScalar(prhs[6]);
    if (step <= 0) mexErrMsgIdAndTxt("aldic:usage", "winstepsize must be positive");
    const int64_t cap = (int64_t)(W / step + 1) * (int64_t)(H / step + 1);
    std::vector<double> buf(5 * (size_t)cap);
    int nx = 0, ny = 0;
    check(aldic_int_search_mg(ctx(), gx, gy, (int)mxGetScalar(prhs[5]), step, &nx, &ny, cap,
                              &buf[0], &buf[cap], &buf[2 * cap], &buf[3 * cap], &buf[4 * cap],
                              nullptr, nullptr));
    // library order x fastest -> MATLAB ny x nx column-major
    for (int o = 0; o < 5 && o < (nlhs > 0 ? nlhs : 1); ++o) {
      plhs[o] = mxCreateDoubleMatrix((size_t)ny, (size_t)nx, mxREAL);
      double *dst = mxGetPr(plhs[o]);
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix)
          dst[iy + (size_t)ix * ny] = buf[(size_t)o * cap + (size_t)iy * nx + ix];
    }
  } else if (c == "computestrain") {
    if (nrhs != 9) mexErrMsgIdAndTxt("aldic:usage", "computestrain takes 8 arguments");
    const int M = (int)mxGetScalar(prhs[1]), N = (int)mxGetScalar(prhs[2]);
    const int method = (int)mxGetScalar(prhs[4]);
    const size_t n = (size_t)M * N;
    if (mxGetNumberOfElements(prhs[7]) != 2 * n) mexErrMsgIdAndTxt("aldic:size", "U is 2*M*N");
    const double *F = nullptr;
    if (method == 0) {
      if (mxGetNumberOfElements(prhs[8]) != 4 * n) mexErrMsgIdAndTxt("aldic:size", "F is 4*M*N");
      F = dbl(prhs[8], "F");
    }
    plhs[0] = mxCreateDoubleMatrix(4 * n, 1, mxREAL);
    mxArray *fin = mxCreateDoubleMatrix(4 * n, 1, mxREAL);
    check(aldic_compute_strain(ctx(), M, N, mxGetScalar(prhs[3]), method, (int)mxGetScalar(prhs[5]),
                               (int)mxGetScalar(prhs[6]), dbl(prhs[7], "U"), F, mxGetPr(plhs[0]),
                               mxGetPr(fin)));
    if (nlhs > 1) plhs[1] = fin; else mxDestroyArray(fin);
  } else if (c == "intsearch") {
    if (nrhs != 8) mexErrMsgIdAndTxt("aldic:usage", "intsearch takes 7 arguments");
    const size_t W = mxGetM(prhs[1]), H = mxGetN(prhs[1]);
    if (mxGetM(prhs[2]) != W || mxGetN(prhs[2]) != H || mxGetClassID(prhs[1]) != mxGetClassID(prhs[2]))
      mexErrMsgIdAndTxt("aldic:size", "f and g differ in size or class");
    int s[2], gx[2], gy[2];
    pair2(prhs[3], "tempSizeOfSearchRegion", s);
    pair2(prhs[4], "gridx", gx);
    pair2(prhs[5], "gridy", gy);
    const int w = (int)mxGetScalar(prhs[6]), step = (int)mxGetScalar(prhs[7]);
    const int dt = img_dtype(prhs[1], "f");
    if (dt == ALDIC_F64) {
      std::vector<double> zeros(W * H, 0.0);  // gradients: not used by the search
      check(aldic_set_fields(ctx(), dbl(prhs[1], "f"), dbl(prhs[2], "g"), zeros.data(),
                             zeros.data(), (int)W, (int)H));
    } else {
      const int roi[4] = {gx[0], gx[1], gy[0], gy[1]};
      check(aldic_set_ref(ctx(), mxGetData(prhs[1]), dt, (int)W, (int)H, roi, nullptr));
      check(aldic_set_def(ctx(), mxGetData(prhs[2]), dt));
    }
    int nx = 0, ny = 0;
    check(aldic_search_dims((int)W, (int)H, gx, gy, w, step, s, &nx, &ny));
    const size_t n = (size_t)nx * ny;
    // the library writes MATLAB's ny x nx column-major arrays directly
    mxArray *o[6];
    for (int k = 0; k < 5; ++k) o[k] = mxCreateDoubleMatrix((size_t)ny, (size_t)nx, mxREAL);
    o[5] = mxCreateDoubleMatrix(n, 2, mxREAL);
    const int rc = aldic_int_search(ctx(), gx, gy, w, step, s, mxGetPr(o[0]), mxGetPr(o[1]),
                                    mxGetPr(o[2]), mxGetPr(o[3]), mxGetPr(o[4]),
                                    nlhs > 5 ? mxGetPr(o[5]) : nullptr);
    give_outputs(o, 6, nlhs, plhs);
    check(rc);
  } else if (c == "subpb2qt") {
    if (nrhs != 8) mexErrMsgIdAndTxt("aldic:usage", "subpb2qt takes 7 arguments");
    const size_t n = mxGetM(prhs[1]), ne = mxGetM(prhs[2]), nd = mxGetNumberOfElements(prhs[3]);
    if (mxGetN(prhs[1]) != 2 || mxGetN(prhs[2]) != 8)
      mexErrMsgIdAndTxt("aldic:size", "coordinatesFEM is n x 2 and elementsFEM ne x 8");
    if (mxGetNumberOfElements(prhs[6]) != 2 * n || mxGetNumberOfElements(prhs[7]) != 4 * n)
      mexErrMsgIdAndTxt("aldic:size", "U is 2n and F is 4n");
    // the library's mesh arrays are MATLAB's column-major n x 2 / ne x 8 as
    // they stand; only the element and Dirichlet indices change type
    const double *cs = dbl(prhs[1], "coordinatesFEM"), *es = dbl(prhs[2], "elementsFEM");
    const double *ds = dbl(prhs[3], "dirichlet");
    std::vector<int32_t> el(8 * ne), dir(nd);
    for (size_t k = 0; k < 8 * ne; ++k) el[k] = (int32_t)es[k];
    for (size_t k = 0; k < nd; ++k) dir[k] = (int32_t)ds[k];
    aldic_qt_mesh *m = nullptr;
    check(aldic_qt_mesh_create((int)n, cs, (int)ne, el.data(), (int)nd, dir.data(), &m));
    plhs[0] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
    const int rc = aldic_qt_subpb2(ctx(), m, mxGetScalar(prhs[4]), mxGetScalar(prhs[5]),
                                   dbl(prhs[6], "U"), dbl(prhs[7], "F"), mxGetPr(plhs[0]));
    aldic_qt_mesh_destroy(m);
    check(rc);
  } else if (c == "frame") {
    if (nrhs != 12) mexErrMsgIdAndTxt("aldic:usage", "frame takes 11 arguments");
    const size_t W = mxGetM(prhs[1]), H = mxGetN(prhs[1]);
    if (mxGetM(prhs[2]) != W || mxGetN(prhs[2]) != H || mxGetClassID(prhs[1]) != mxGetClassID(prhs[2]))
      mexErrMsgIdAndTxt("aldic:size", "ImgRef and ImgDef differ in size or class");
    aldic_frame_params p;
    std::memset(&p, 0, sizeof p);
    p.winsize = (int)mxGetScalar(prhs[3]);
    p.step = (int)mxGetScalar(prhs[4]);
    pair2(prhs[5], "tempSizeOfSearchRegion", p.search);
    pair2(prhs[6], "gridx", p.gridx);
    pair2(prhs[7], "gridy", p.gridy);
    p.tol = mxGetScalar(prhs[8]);
    p.mu = 1e-3;
    p.beta = 0.0;
    p.n_admm = (int)mxGetScalar(prhs[9]);
    p.tol2 = 0.0;  // every one of the nADMM steps runs; stats holds UpdateY of each
    p.precision = ALDIC_FP64;
    p.subpb2_fd = mxGetScalar(prhs[10]) == 1.0;
    p.smooth = mxGetScalar(prhs[11]) != 0.0;
    p.use_graph = 1;
    p.init = ALDIC_INIT_SEARCH;
    const int dt = img_dtype(prhs[1], "ImgRef");
    const int roi[4] = {p.gridx[0], p.gridx[1], p.gridy[0], p.gridy[1]};
    check(aldic_set_ref(ctx(), mxGetData(prhs[1]), dt, (int)W, (int)H, roi, nullptr));
    check(aldic_set_def(ctx(), mxGetData(prhs[2]), dt));
    int M = 0, N = 0;
    check(aldic_frame_dims(ctx(), &p, &M, &N));
    const size_t n = (size_t)M * N;
    // x0, y0 as MeshSetUp.m's M x N arrays (x index first: node k = i + M j,
    // the library's x-fastest order)
    mxArray *o[6];
    o[0] = mxCreateDoubleMatrix((size_t)M, (size_t)N, mxREAL);
    o[1] = mxCreateDoubleMatrix((size_t)M, (size_t)N, mxREAL);
    o[2] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
    o[3] = mxCreateDoubleMatrix(4 * n, 1, mxREAL);
    mwSize d1[2] = {n, 1};
    o[4] = mxCreateNumericArray(2, d1, mxINT32_CLASS, mxREAL);
    aldic_frame_stats st;
    std::memset(&st, 0, sizeof st);
    const int rc = aldic_frame(ctx(), &p, mxGetPr(o[0]), mxGetPr(o[1]), mxGetPr(o[2]),
                               mxGetPr(o[3]), (int32_t *)mxGetData(o[4]), &st);
    o[5] = mxCreateDoubleMatrix(1, 2 + (size_t)st.admm_steps, mxREAL);
    double *sv = mxGetPr(o[5]);
    sv[0] = st.beta;
    sv[1] = st.bad_icgn;
    for (int a = 0; a < st.admm_steps; ++a) sv[2 + a] = st.update_y[a];
    give_outputs(o, 6, nlhs, plhs);
    check(rc);
  } else {
    mexErrMsgIdAndTxt("aldic:usage", "unknown command '%s'", cmd);
  }
}
