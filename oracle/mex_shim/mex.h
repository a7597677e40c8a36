/*
 * mex.h -- minimal, project-written stand-in for the MATLAB MEX API.
 *
 * TEST INFRASTRUCTURE ONLY.  MATLAB is not installed here, so this header
 * declares just the mxArray calls that the reference's ba_interp2.cpp and the
 * project's own MEX gateways use, with MATLAB's documented semantics:
 * column-major numeric arrays, mexErrMsgTxt aborting the call (here: a C++
 * exception that the test harness catches).
 */
#ifndef ALDIC_MEX_SHIM_H
#define ALDIC_MEX_SHIM_H
#include <stddef.h>

typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7,
               mxINT32_CLASS = 12, mxUINT8_CLASS = 9, mxUINT16_CLASS = 11,
               mxCHAR_CLASS = 4, mxSTRUCT_CLASS = 2 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag mxArray;

#ifdef __cplusplus
extern "C" {
#endif
const mwSize *mxGetDimensions(const mxArray *a);
mwSize mxGetNumberOfDimensions(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
int mxIsDouble(const mxArray *a);
int mxIsSingle(const mxArray *a);
int mxIsUint8(const mxArray *a);
int mxIsUint16(const mxArray *a);
int mxIsInt32(const mxArray *a);
int mxIsStruct(const mxArray *a);
mxClassID mxGetClassID(const mxArray *a);
void *mxGetData(const mxArray *a);
double *mxGetPr(const mxArray *a);
double mxGetScalar(const mxArray *a);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity c);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray *mxCreateDoubleScalar(double v);
mxArray *mxGetField(const mxArray *s, mwIndex i, const char *name);
void mxDestroyArray(mxArray *a);
void mexErrMsgTxt(const char *msg);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
int mexAtExit(void (*fn)(void));
void mexLock(void);

/* harness-side helpers (not part of the MATLAB API) */
mxArray *shim_wrap(mxClassID cls, mwSize ndim, const mwSize *dims, void *data);
mxArray *shim_struct(int nfields, const char **names, mxArray **values);
const char *shim_last_error(void);
#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#else
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#endif
#endif
