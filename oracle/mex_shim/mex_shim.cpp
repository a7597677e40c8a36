/*
 * mex_shim.cpp -- implementation of the project-written mex.h stand-in.
 * TEST INFRASTRUCTURE ONLY (see mex.h).
 */
#include "mex.h"

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

struct mxArray_tag {
  mxClassID cls = mxUNKNOWN_CLASS;
  std::vector<mwSize> dims;
  void *data = nullptr;
  bool owns = false;
  std::vector<std::string> names;      // struct fields
  std::vector<mxArray *> fields;
};

static thread_local std::string g_err;

static size_t elem_size(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: return 8;
    case mxSINGLE_CLASS: return 4;
    case mxINT32_CLASS: return 4;
    case mxUINT16_CLASS: return 2;
    case mxUINT8_CLASS: return 1;
    case mxCHAR_CLASS: return 2;
    default: return 0;
  }
}

extern "C" {
const mwSize *mxGetDimensions(const mxArray *a) { return a->dims.data(); }
mwSize mxGetNumberOfDimensions(const mxArray *a) { return a->dims.size(); }
size_t mxGetNumberOfElements(const mxArray *a) {
  size_t n = 1;
  for (auto d : a->dims) n *= d;
  return n;
}
size_t mxGetM(const mxArray *a) { return a->dims.empty() ? 0 : a->dims[0]; }
size_t mxGetN(const mxArray *a) {
  size_t n = 1;
  for (size_t i = 1; i < a->dims.size(); ++i) n *= a->dims[i];
  return n;
}
int mxIsDouble(const mxArray *a) { return a->cls == mxDOUBLE_CLASS; }
int mxIsSingle(const mxArray *a) { return a->cls == mxSINGLE_CLASS; }
int mxIsUint8(const mxArray *a) { return a->cls == mxUINT8_CLASS; }
int mxIsUint16(const mxArray *a) { return a->cls == mxUINT16_CLASS; }
int mxIsInt32(const mxArray *a) { return a->cls == mxINT32_CLASS; }
int mxIsStruct(const mxArray *a) { return a->cls == mxSTRUCT_CLASS; }
mxClassID mxGetClassID(const mxArray *a) { return a->cls; }
void *mxGetData(const mxArray *a) { return a->data; }
double *mxGetPr(const mxArray *a) { return (double *)a->data; }
double mxGetScalar(const mxArray *a) {
  switch (a->cls) {
    case mxDOUBLE_CLASS: return *(double *)a->data;
    case mxSINGLE_CLASS: return *(float *)a->data;
    case mxINT32_CLASS: return *(int *)a->data;
    default: return 0.0;
  }
}
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity) {
  mxArray *a = new mxArray_tag();
  a->cls = cls;
  a->dims.assign(dims, dims + ndim);
  size_t n = mxGetNumberOfElements(a);
  a->data = std::calloc(n ? n : 1, elem_size(cls));
  a->owns = true;
  return a;
}
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
  mwSize d[2] = {m, n};
  return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, c);
}
mxArray *mxCreateDoubleScalar(double v) {
  mxArray *a = mxCreateDoubleMatrix(1, 1, mxREAL);
  *(double *)a->data = v;
  return a;
}
mxArray *mxGetField(const mxArray *s, mwIndex, const char *name) {
  if (!s || s->cls != mxSTRUCT_CLASS) return nullptr;
  for (size_t i = 0; i < s->names.size(); ++i)
    if (s->names[i] == name) return s->fields[i];
  return nullptr;
}
void mxDestroyArray(mxArray *a) {
  if (!a) return;
  if (a->owns) std::free(a->data);
  delete a;
}
void mexErrMsgTxt(const char *msg) {
  g_err = msg;
  throw std::runtime_error(msg);
}
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = std::string(id) + ": " + buf;
  throw std::runtime_error(g_err);
}
int mexAtExit(void (*)(void)) { return 0; }
void mexLock(void) {}

mxArray *shim_wrap(mxClassID cls, mwSize ndim, const mwSize *dims, void *data) {
  mxArray *a = new mxArray_tag();
  a->cls = cls;
  a->dims.assign(dims, dims + ndim);
  a->data = data;
  a->owns = false;
  return a;
}
mxArray *shim_struct(int nfields, const char **names, mxArray **values) {
  mxArray *a = new mxArray_tag();
  a->cls = mxSTRUCT_CLASS;
  a->dims = {1, 1};
  for (int i = 0; i < nfields; ++i) {
    a->names.push_back(names[i]);
    a->fields.push_back(values[i]);
  }
  return a;
}
const char *shim_last_error(void) { return g_err.c_str(); }
}
