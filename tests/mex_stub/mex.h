/* Minimal stand-in for MATLAB's mex.h (test infrastructure): declares just what the
 * MEX gateways in ctsim_b200/mex/ use, so that they can be compiled, and linked with
 * mex_fake.c and called, on a machine without MATLAB. */
#ifndef CTSIM_TEST_MEX_STUB_H
#define CTSIM_TEST_MEX_STUB_H
#include <stdbool.h>
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxSINGLE_CLASS = 7 } mxClassID;
typedef enum { mxREAL = 0 } mxComplexity;
void *mxGetData(const mxArray *);
int mxIsChar(const mxArray *);
int mxGetString(const mxArray *, char *, mwSize);
size_t mxGetM(const mxArray *);
size_t mxGetN(const mxArray *);
bool mxIsDouble(const mxArray *);
bool mxIsComplex(const mxArray *);
bool mxIsSingle(const mxArray *);
bool mxIsLogical(const mxArray *);
mwSize mxGetNumberOfDimensions(const mxArray *);
const mwSize *mxGetDimensions(const mxArray *);
mxArray *mxCreateNumericArray(mwSize, const mwSize *, mxClassID, mxComplexity);
void mexErrMsgTxt(const char *);
int mexPrintf(const char *, ...);
#endif
