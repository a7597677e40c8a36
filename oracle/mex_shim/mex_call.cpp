/*
 * mex_call.cpp -- C entry that runs a compiled mexFunction the way MATLAB
 * would: wraps caller-owned column-major buffers as mxArrays, calls
 * mexFunction, copies plhs[0] back and turns mexErrMsgTxt into a return code.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <cstring>
#include <stdexcept>

#include "mex.h"

extern "C" int shim_call_mex(int nlhs, int nrhs, const int *cls, const int *ndims,
                             const long long *dims, void **datas, void *out,
                             size_t out_bytes, long long *out_dims, int *out_ndim) {
  mxArray *prhs[16];
  mxArray *plhs[4] = {nullptr, nullptr, nullptr, nullptr};
  int rc = 0;
  const long long *dp = dims;
  for (int i = 0; i < nrhs; ++i) {
    mwSize d[8];
    for (int k = 0; k < ndims[i]; ++k) d[k] = (mwSize)dp[k];
    dp += ndims[i];
    prhs[i] = shim_wrap((mxClassID)cls[i], (mwSize)ndims[i], d, datas[i]);
  }
  try {
    mexFunction(nlhs, plhs, nrhs, (const mxArray **)prhs);
    if (nlhs > 0 && plhs[0]) {
      size_t n = mxGetNumberOfElements(plhs[0]);
      size_t es = mxIsDouble(plhs[0]) ? 8 : 4;
      if (n * es > out_bytes) rc = -2;
      else std::memcpy(out, mxGetData(plhs[0]), n * es);
      *out_ndim = (int)mxGetNumberOfDimensions(plhs[0]);
      for (int k = 0; k < *out_ndim && k < 8; ++k) out_dims[k] = (long long)mxGetDimensions(plhs[0])[k];
    }
  } catch (const std::exception &) {
    rc = -1;
  }
  for (int i = 0; i < nrhs; ++i) mxDestroyArray(prhs[i]);
  for (int i = 0; i < 4; ++i) mxDestroyArray(plhs[i]);
  return rc;
}

// Several outputs: outs[i] receives plhs[i] (out_bytes[i] capacity).
extern "C" int shim_call_mex_n(int nlhs, int nrhs, const int *cls, const int *ndims,
                               const long long *dims, void **datas, void **outs,
                               const size_t *out_bytes) {
  mxArray *prhs[16];
  mxArray *plhs[8] = {nullptr};
  int rc = 0;
  const long long *dp = dims;
  for (int i = 0; i < nrhs; ++i) {
    mwSize d[8];
    for (int k = 0; k < ndims[i]; ++k) d[k] = (mwSize)dp[k];
    dp += ndims[i];
    prhs[i] = shim_wrap((mxClassID)cls[i], (mwSize)ndims[i], d, datas[i]);
  }
  try {
    mexFunction(nlhs, plhs, nrhs, (const mxArray **)prhs);
    for (int o = 0; o < nlhs && o < 8; ++o) {
      if (!plhs[o]) continue;
      size_t n = mxGetNumberOfElements(plhs[o]);
      size_t es = mxIsDouble(plhs[o]) ? 8 : 4;
      if (n * es > out_bytes[o]) rc = -2;
      else std::memcpy(outs[o], mxGetData(plhs[o]), n * es);
    }
  } catch (const std::exception &) {
    rc = -1;
  }
  for (int i = 0; i < nrhs; ++i) mxDestroyArray(prhs[i]);
  for (int i = 0; i < 8; ++i) mxDestroyArray(plhs[i]);
  return rc;
}
