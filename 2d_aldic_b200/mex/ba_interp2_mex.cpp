// ba_interp2_mex.cpp -- drop-in MEX gateway for the reference's ba_interp2.
//
//     mex -R2018a ba_interp2_mex.cpp -I<repo>/include -L<repo>/2d_aldic_b200 \
//         -laldic_b200 -output ba_interp2
//
// Same interface as ba_interp2.cpp:318-335: Z = ba_interp2(F, X, Y, [method])
// with F an M x N (x P) double or single image, X indexing columns and Y
// rows (1-based), Z of size(X) x P, clamp-to-edge Keys bicubic.  The argument
// checks and their messages are the reference's, so callers see the same
// errors; the sampling runs on the GPU (libaldic_b200) and is bit-identical
// to the reference's CPU results.
#include <mex.h>

#include "aldic_b200.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  if ((nrhs != 3) && (nrhs != 4))
    mexErrMsgTxt("Wrong number of input arguments for Z = ba_interp2(F, X, Y, [method])");
  if (nlhs > 1)
    mexErrMsgTxt("Wrong number of output arguments for Z = ba_interp2(F, X, Y, [method])");
  const mxArray *F = prhs[0], *X = prhs[1], *Y = prhs[2];
  const bool dbl = mxIsDouble(F) && mxIsDouble(X) && mxIsDouble(Y);
  const bool sgl = mxIsSingle(F) && mxIsSingle(X) && mxIsSingle(Y);
  if (!dbl && !sgl)
    mexErrMsgTxt("ba_interp2 takes only double or single arguments for IMG,X,Y, and all must "
                 "have the same class");
  const mwSize nx = mxGetNumberOfDimensions(X), nf = mxGetNumberOfDimensions(F);
  if (nx != mxGetNumberOfDimensions(Y)) mexErrMsgTxt("X, Y should have the same size");
  if (nx + nf - 2 > 50) mexErrMsgTxt("Can't have that many dimensions in interpolated data.");
  const mwSize *fd = mxGetDimensions(F), *xd = mxGetDimensions(X), *yd = mxGetDimensions(Y);
  mwSize od[50];
  for (mwSize i = 0; i < nx; ++i) {
    if (xd[i] != yd[i]) mexErrMsgTxt("X, Y should have the same size");
    od[i] = xd[i];
  }
  int64_t P = 1;
  for (mwSize i = 2; i < nf; ++i) {
    od[nx + i - 2] = fd[i];
    P *= (int64_t)fd[i];
  }
  plhs[0] = mxCreateNumericArray(nx + nf - 2, od, sgl ? mxSINGLE_CLASS : mxDOUBLE_CLASS, mxREAL);
  const int64_t M = (int64_t)fd[0], N = (int64_t)(nf > 1 ? fd[1] : 1);
  const int64_t n = (int64_t)mxGetNumberOfElements(X);
  if (n == 0 || M == 0 || N == 0) return;
  int rc = dbl ? aldic_ba_interp2_f64((const double *)mxGetData(F), M, N, P,
                                      (const double *)mxGetData(X), (const double *)mxGetData(Y),
                                      n, (double *)mxGetData(plhs[0]), nullptr)
               : aldic_ba_interp2_f32((const float *)mxGetData(F), M, N, P,
                                      (const float *)mxGetData(X), (const float *)mxGetData(Y), n,
                                      (float *)mxGetData(plhs[0]), nullptr);
  if (rc != ALDIC_OK) mexErrMsgIdAndTxt("aldic:ba_interp2", "%s", aldic_last_error());
}
