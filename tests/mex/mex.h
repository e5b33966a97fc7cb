/*
 * mex.h -- TEST-ONLY stand-in for the MATLAB C API (MATLAB and GNU Octave are
 * not installed where this library is built and tested).  It declares the
 * few mxArray / mex functions that matlab/starmap_solver_mex.c calls, with
 * their published names and meanings, over plain C arrays
 * (tests/mex/mex_stub.c), so that the gateway can be compiled, linked
 * against libstarmap_gpu.so and called from the test suite.  It is not
 * MATLAB's header and is never used to build the gateway for MATLAB.
 */
#ifndef SMG_TEST_MEX_H
#define SMG_TEST_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxCELL_CLASS = 1, mxSTRUCT_CLASS = 2, mxCHAR_CLASS = 4, mxDOUBLE_CLASS = 6 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

int mxIsDouble(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsSparse(const mxArray* a);
int mxIsCell(const mxArray* a);
int mxIsStruct(const mxArray* a);
int mxIsChar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize len);
size_t mxGetNumberOfElements(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
double* mxGetPr(const mxArray* a);
double mxGetScalar(const mxArray* a);
mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name);
mxArray* mxGetCell(const mxArray* c, mwIndex i);
void mxSetCell(mxArray* c, mwIndex i, mxArray* v);
mxArray* mxCreateCellMatrix(mwSize m, mwSize n);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cx);
mxArray* mxCreateDoubleScalar(double v);
void* mxMalloc(size_t n);
void mxFree(void* p);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

#ifdef __cplusplus
}
#endif

#endif
