/* Test-side implementation of the MEX API functions that the gateways in ctsim_b200/mex/
 * call (test infrastructure, MATLAB is not available here).  An mxArray is a class tag,
 * its dimensions and its data; mexErrMsgTxt records the message and jumps back to
 * fake_call, as MATLAB's error leaves the MEX function.  Linked with one gateway into a
 * shared library that the tests drive through ctypes. */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

enum { kDouble = 0, kSingle = 1, kInt32 = 2, kLogical = 3, kChar = 4 };

struct mxArray_tag {
    int cls;
    mwSize ndim;
    mwSize dims[4];
    void *data;
};

static jmp_buf g_jmp;
static char g_err[512];
static char g_out[8192];
static size_t g_out_len;

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

static size_t elem_size(int cls) { return cls == kDouble ? 8 : cls == kSingle || cls == kInt32 ? 4 : 1; }

static size_t numel(const mxArray *a) {
    size_t n = 1;
    for (mwSize i = 0; i < a->ndim; i++) n *= a->dims[i];
    return n;
}

/* An array of class cls with ndim (<= 4) dimensions; its data (copied) or zeros. */
mxArray *fake_array(int cls, int ndim, const size_t *dims, const void *data) {
    mxArray *a = calloc(1, sizeof(mxArray));
    a->cls = cls;
    a->ndim = (mwSize)ndim;
    for (int i = 0; i < ndim; i++) a->dims[i] = dims[i];
    size_t bytes = numel(a) * elem_size(cls) + (cls == kChar ? 1 : 0);
    a->data = calloc(1, bytes ? bytes : 1);
    if (data) memcpy(a->data, data, numel(a) * elem_size(cls));
    return a;
}
void *fake_data(mxArray *a) { return a->data; }
size_t fake_numel(mxArray *a) { return numel(a); }
int fake_class(mxArray *a) { return a->cls; }
void fake_free(mxArray *a) {
    if (!a) return;
    free(a->data);
    free(a);
}
const char *fake_error(void) { return g_err; }
const char *fake_output(void) { return g_out; }

/* Runs mexFunction; returns 0, or 1 when it raised an error (message in fake_error). */
int fake_call(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs) {
    g_err[0] = 0;
    g_out[0] = 0;
    g_out_len = 0;
    if (setjmp(g_jmp)) return 1;
    mexFunction(nlhs, plhs, nrhs, prhs);
    return 0;
}

void *mxGetData(const mxArray *a) { return a->data; }
int mxIsChar(const mxArray *a) { return a->cls == kChar; }
int mxGetString(const mxArray *a, char *buf, mwSize n) {
    if (a->cls != kChar || n == 0) return 1;
    size_t len = numel(a);
    if (len + 1 > n) return 1;
    memcpy(buf, a->data, len);
    buf[len] = 0;
    return 0;
}
size_t mxGetM(const mxArray *a) { return a->ndim ? a->dims[0] : 0; }
size_t mxGetN(const mxArray *a) {
    size_t n = 1;
    for (mwSize i = 1; i < a->ndim; i++) n *= a->dims[i];
    return n;
}
bool mxIsDouble(const mxArray *a) { return a->cls == kDouble; }
bool mxIsComplex(const mxArray *a) { (void)a; return false; }
bool mxIsSingle(const mxArray *a) { return a->cls == kSingle; }
bool mxIsLogical(const mxArray *a) { return a->cls == kLogical; }
mwSize mxGetNumberOfDimensions(const mxArray *a) { return a->ndim; }
const mwSize *mxGetDimensions(const mxArray *a) { return a->dims; }
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity c) {
    (void)c;
    size_t d[4];
    for (mwSize i = 0; i < ndim && i < 4; i++) d[i] = dims[i];
    return fake_array(cls == mxSINGLE_CLASS ? kSingle : kDouble, (int)ndim, d, NULL);
}
void mexErrMsgTxt(const char *msg) {
    snprintf(g_err, sizeof(g_err), "%s", msg);
    longjmp(g_jmp, 1);
}
int mexPrintf(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(g_out + g_out_len, sizeof(g_out) - g_out_len, fmt, ap);
    va_end(ap);
    if (n > 0) g_out_len += (size_t)n < sizeof(g_out) - g_out_len ? (size_t)n : sizeof(g_out) - g_out_len - 1;
    return n;
}
