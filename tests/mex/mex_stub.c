/*
 * mex_stub.c -- TEST-ONLY implementation of the MATLAB C API subset declared
 * in tests/mex/mex.h, over plain C arrays, plus the entry points the tests
 * call through ctypes to build arguments, call mexFunction and read its
 * outputs.  mexErrMsgIdAndTxt returns to stub_call with longjmp, as MATLAB
 * unwinds a failing MEX call.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
    int cls;
    char* str;
    mwSize ndim;
    mwSize dims[8];
    double* pr;
    mxArray** cells;
    int nfields;
    char** names;
    mxArray** values;
};

static jmp_buf g_jump;
static char g_err[2048];
static char g_err_id[256];

static size_t numel(const mxArray* a) {
    size_t n = 1;
    for (mwSize k = 0; k < a->ndim; ++k) n *= a->dims[k];
    return n;
}

int mxIsDouble(const mxArray* a) { return a && a->cls == mxDOUBLE_CLASS; }
int mxIsComplex(const mxArray* a) { (void)a; return 0; }
int mxIsSparse(const mxArray* a) { (void)a; return 0; }
int mxIsCell(const mxArray* a) { return a && a->cls == mxCELL_CLASS; }
int mxIsStruct(const mxArray* a) { return a && a->cls == mxSTRUCT_CLASS; }
int mxIsChar(const mxArray* a) { return a && a->cls == mxCHAR_CLASS; }
int mxGetString(const mxArray* a, char* buf, mwSize len) {
    if (!a || a->cls != mxCHAR_CLASS || !len) return 1;
    const size_t n = strlen(a->str);
    memcpy(buf, a->str, n < len ? n : len - 1);
    buf[n < len ? n : len - 1] = '\0';
    return n < len ? 0 : 1;
}
size_t mxGetNumberOfElements(const mxArray* a) { return numel(a); }
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) { return numel(a) / (a->dims[0] ? a->dims[0] : 1); }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->ndim; }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims; }
double* mxGetPr(const mxArray* a) { return a->pr; }
double mxGetScalar(const mxArray* a) { return (a && a->pr && numel(a) > 0) ? a->pr[0] : 0.0; }

mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name) {
    if (!s || s->cls != mxSTRUCT_CLASS || i != 0) return NULL;
    for (int k = 0; k < s->nfields; ++k)
        if (strcmp(s->names[k], name) == 0) return s->values[k];
    return NULL;
}

mxArray* mxGetCell(const mxArray* c, mwIndex i) { return (c && i < numel(c)) ? c->cells[i] : NULL; }
void mxSetCell(mxArray* c, mwIndex i, mxArray* v) { c->cells[i] = v; }

static mxArray* make(int cls, mwSize ndim, const mwSize* dims) {
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    a->cls = cls;
    a->ndim = ndim < 2 ? 2 : ndim;
    a->dims[0] = a->dims[1] = 1;
    for (mwSize k = 0; k < ndim && k < 8; ++k) a->dims[k] = dims[k];
    if (cls == mxDOUBLE_CLASS) a->pr = (double*)calloc(numel(a) ? numel(a) : 1, sizeof(double));
    if (cls == mxCELL_CLASS) a->cells = (mxArray**)calloc(numel(a) ? numel(a) : 1, sizeof(mxArray*));
    return a;
}

mxArray* mxCreateCellMatrix(mwSize m, mwSize n) {
    mwSize d[2] = {m, n};
    return make(mxCELL_CLASS, 2, d);
}

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cx) {
    (void)cx;
    return make(cls, ndim, dims);
}

mxArray* mxCreateDoubleScalar(double v) {
    mwSize d[2] = {1, 1};
    mxArray* a = make(mxDOUBLE_CLASS, 2, d);
    a->pr[0] = v;
    return a;
}

void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void* p) { free(p); }

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    snprintf(g_err_id, sizeof g_err_id, "%s", id);
    longjmp(g_jump, 1);
}

/* ---- entry points of the test harness ---------------------------------- */
mxArray* stub_double(mwSize ndim, const mwSize* dims, const double* data) {
    mxArray* a = make(mxDOUBLE_CLASS, ndim, dims);
    if (data) memcpy(a->pr, data, numel(a) * sizeof(double));
    return a;
}

mxArray* stub_cell(mwSize n) { return mxCreateCellMatrix(1, n); }

mxArray* stub_string(const char* s) {
    mwSize d[2] = {1, 1};
    mxArray* a = make(mxCHAR_CLASS, 2, d);
    d[1] = strlen(s);
    a->dims[1] = d[1];
    a->str = (char*)malloc(d[1] + 1);
    strcpy(a->str, s);
    return a;
}

mxArray* stub_struct(void) {
    mwSize d[2] = {1, 1};
    mxArray* a = make(mxSTRUCT_CLASS, 2, d);
    a->names = (char**)calloc(64, sizeof(char*));
    a->values = (mxArray**)calloc(64, sizeof(mxArray*));
    return a;
}

int stub_struct_set(mxArray* s, const char* name, mxArray* v) {
    if (s->nfields >= 64) return -1;
    s->names[s->nfields] = (char*)malloc(strlen(name) + 1);
    strcpy(s->names[s->nfields], name);
    s->values[s->nfields++] = v;
    return 0;
}

/* 0: mexFunction returned; 1: it raised an error (stub_error / stub_error_id) */
int stub_call(int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
    g_err[0] = g_err_id[0] = '\0';
    if (setjmp(g_jump)) return 1;
    mexFunction(nlhs, plhs, nrhs, prhs);
    return 0;
}

const char* stub_error(void) { return g_err; }
const char* stub_error_id(void) { return g_err_id; }
