/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * The reference's own CUDA FDK backprojection (geom/fdk_cuda/cbct_back_pd.c, the
 * kernels and host driver that its MEX gateway geom/fdk_cuda/cbct_back_pd_cuda.cu
 * includes) compiled unmodified for sm_100a from the read-only checkout, with the
 * stand-in mex.h of tests/mex_stub.  A timing baseline beside this project's kernels.
 *
 *   refgpu_back_pd   cbct_back_pd_gpu  geom/fdk_cuda/cbct_back_pd.c:230
 *
 * Host pointers, synchronous; the reference's error handler (book.h) exits the
 * process on a CUDA error.
 */
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include "mex.h"
// the MATLAB allocation calls that ct_def.h's helpers name, and definitions of the
// stand-in header's calls that the drivers reach (printing and errors only)
void *mxCalloc(size_t n, size_t size);
void mxFree(void *p);
#include "ct_def.h"
#include "book.h"

#include "cbct_back_pd.c"

extern "C" bool refgpu_back_pd(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                               int nu, int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd,
                               int noviews, double *betas, float *couchz, int detector_type, float *image,
                               float *proj, bool *map, bool off_boundary) {
    return cbct_back_pd_gpu(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd, noviews,
                            betas, couchz, detector_type, image, proj, map, off_boundary);
}

void *mxCalloc(size_t n, size_t size) { return calloc(n, size); }
void mxFree(void *p) { free(p); }
int mexPrintf(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    const int r = vprintf(fmt, ap);
    va_end(ap);
    return r;
}
void mexErrMsgTxt(const char *msg) {
    fprintf(stderr, "%s\n", msg);
    exit(EXIT_FAILURE);
}
size_t mxGetM(const mxArray *) { return 0; }
size_t mxGetN(const mxArray *) { return 0; }
int mxGetString(const mxArray *, char *, mwSize) { return 1; }
