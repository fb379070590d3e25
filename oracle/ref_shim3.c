/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Compiles the reference's arc-detector variants of the distance-driven pair,
 * geom/cbct/cbct_proj3.c and geom/cbct/cbct_back3.c (detector_type 2, "special arc
 * panel"), unmodified from the read-only reference checkout, and exposes proj,dd and
 * back,dd through the same zero-filled, input-preserving C ABI as ref_shim.c.  No
 * MEX gateway of the reference includes these two files; they are the only source
 * of the arc-detector footprints.
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

#include "cbct_proj3.c"
#include "cbct_back3.c"

/* kind: 0 proj,dd  2 back,dd */
int ref3_cbct_call(int kind, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                   int nu, int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd,
                   int noviews, const double *betas, const float *couchz, int detector_type,
                   const float *in, float *out, const bool *map)
{
    long nxyz = (long)nx * ny * nz, nsino = (long)nu * nv * noviews;
    long nin = kind == 0 ? nxyz : nsino, nout = kind == 0 ? nsino : nxyz;
    float *copy = (float *)malloc(sizeof(float) * (nin > 0 ? nin : 1));
    bool ok = false;
    if (!copy) return 0;
    memcpy(copy, in, sizeof(float) * nin);
    memset(out, 0, sizeof(float) * nout);
    if (kind == 0)
        ok = cbct_proj_dd(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd, noviews,
                          (double *)betas, (float *)couchz, detector_type, copy, out, (bool *)map);
    else if (kind == 2)
        ok = cbct_back_dd(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd, noviews,
                          (double *)betas, (float *)couchz, detector_type, out, copy, (bool *)map);
    free(copy);
    return ok ? 1 : 0;
}
