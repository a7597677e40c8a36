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
  } else {
    mexErrMsgIdAndTxt("aldic:usage", "unknown command '%s'", cmd);
  }
}
