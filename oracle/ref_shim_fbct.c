/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Compiles the reference's 2-D fan-beam projectors, geom/fbct/fbct_proj.c and
 * geom/fbct/fbct_back.c, unmodified from the read-only reference checkout, and
 * exposes the distance-driven and separable-footprint pair with zero-filled
 * outputs (the MEX gateway's mxCreateNumericArray, geom/fbct/fbct_geom_mex.c:110).
 */
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>

#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef min
#define min(a, b) (((a) < (b)) ? (a) : (b))
#endif

#include "fbct_proj.c"
#include "fbct_back.c"

/* kind: 0 proj,dd  1 proj,tf  2 back,dd  3 back,tf */
int ref_fbct_call(int kind, int nx, int ny, float dx, float dy, float ox, float oy, int nu, float du, float ou,
                  float sad, float add, float sdd, int noviews, const double *betas, int det, const float *in,
                  float *out)
{
    long nxy = (long)nx * ny, nsino = (long)nu * noviews;
    long nin = kind <= 1 ? nxy : nsino, nout = kind <= 1 ? nsino : nxy;
    float *copy = (float *)malloc(sizeof(float) * (nin > 0 ? nin : 1));
    bool ok = false;
    if (!copy) return 0;
    memcpy(copy, in, sizeof(float) * nin);
    memset(out, 0, sizeof(float) * nout);
    switch (kind) {
    case 0: ok = fbct_proj_dd(nx, ny, dx, dy, ox, oy, nu, du, ou, sad, add, sdd, noviews, (double *)betas, det, copy, out); break;
    case 1: ok = fbct_proj_tf(nx, ny, dx, dy, ox, oy, nu, du, ou, sad, add, sdd, noviews, (double *)betas, det, copy, out); break;
    case 2: ok = fbct_back_dd(nx, ny, dx, dy, ox, oy, nu, du, ou, sad, add, sdd, noviews, (double *)betas, det, out, copy); break;
    case 3: ok = fbct_back_tf(nx, ny, dx, dy, ox, oy, nu, du, ou, sad, add, sdd, noviews, (double *)betas, det, out, copy); break;
    }
    free(copy);
    return ok ? 1 : 0;
}
