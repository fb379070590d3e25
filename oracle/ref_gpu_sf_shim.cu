/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * The reference's own CUDA separable-footprint pair (geom/sf_cuda/cbct_sf_proj.c and
 * cbct_sf_back.c, the kernels and host drivers that its MEX gateway
 * geom/sf_cuda/cbct_sf_cuda.cu includes) compiled unmodified for sm_100a from the
 * read-only checkout (-I to its directory; nothing is copied into this repository),
 * with the stand-in mex.h of tests/mex_stub.  A timing baseline on the same B200 beside
 * this project's kernels; not a parity target (the reference's CPU C is).
 *
 *   refgpu_proj_tf   cbct_proj_tf_gpu  geom/sf_cuda/cbct_sf_proj.c:443
 *   refgpu_back_tf   cbct_back_tf_gpu  geom/sf_cuda/cbct_sf_back.c:334
 *
 * Host pointers, synchronous; the reference's error handler (book.h) exits the process
 * on a CUDA error.  Its kernels launch nv (forward) and nz (backward) threads per block,
 * so both must be at most 1024.
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

#include "cbct_sf_back.c"
#include "cbct_sf_proj.c"

extern "C" bool refgpu_proj_tf(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                               int nu, int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd,
                               int noviews, double *betas, float *couchz, int detector_type, float *image,
                               float *proj, bool *map) {
    return cbct_proj_tf_gpu(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd, noviews,
                            betas, couchz, detector_type, image, proj, map);
}

extern "C" bool refgpu_back_tf(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                               int nu, int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd,
                               int noviews, double *betas, float *couchz, int detector_type, float *image,
                               float *proj, bool *map) {
    return cbct_back_tf_gpu(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd, noviews,
                            betas, couchz, detector_type, image, proj, map);
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
