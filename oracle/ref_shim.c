/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Compiles the reference's own, unmodified CPU projectors
 * (geom/cbct/cbct_proj.c, geom/cbct/cbct_back.c, geom/cbct/cbct_back_var.c)
 * straight from the read-only reference checkout (the include path is given by
 * oracle/Makefile), and wraps them in a small C ABI that:
 *
 *   - never mutates caller inputs: the reference back-projectors scale their
 *     sinogram argument in place (geom/cbct/cbct_back.c:196-214 for `back,dd`,
 *     :437-455 for `back,tf`), so the wrappers hand them a private copy;
 *   - zero-fills outputs first, as the MEX gateway's mxCreateNumericArray does
 *     (geom/cbct/cbct_geom_mex.c:117, :230), because the reference accumulates
 *     with `+=`;
 *   - adds a pthread harness over contiguous view chunks for the CPU baseline
 *     (forward: disjoint view slices; backward: one image per thread, summed).
 *
 * The include order mirrors geom/cbct/cbct_geom_mex.c:7-9: cbct_proj.c defines
 * FOOTPRINT_SIZE_U/V (= 10) which cbct_back.c relies on.
 */
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>
#include <pthread.h>

/* The two macros geom/cbct/ct_def.h:11-17 supplies (ct_def.h itself needs mex.h). */
#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef min
#define min(a, b) (((a) < (b)) ? (a) : (b))
#endif

#include "cbct_proj.c"
#include "cbct_back.c"
#include "cbct_back_var.c"

/* kind: 0 proj,dd  1 proj,tf  2 back,dd  3 back,tf  4 back,pd  5 back,hpd  6 back,var */
typedef struct {
    int kind;
    int nx, ny, nz;
    float dx, dy, dz, ox, oy, oz;
    int nu, nv;
    float du, dv, ou, ov, sad, add, sdd;
    int noviews;
    const double *betas;
    const float *couchz;
    int detector_type;
    const float *in;
    float *out;
    const bool *map;
} ref_call;

static int run_one(const ref_call *c)
{
    long nxyz = (long)c->nx * c->ny * c->nz;
    long nsino = (long)c->nu * c->nv * c->noviews;
    bool ok = false;
    double *betas = (double *)c->betas;
    float *couchz = (float *)c->couchz;
    bool *map = (bool *)c->map;
    if (c->kind <= 1) {
        float *img = (float *)malloc(sizeof(float) * (nxyz > 0 ? nxyz : 1));
        if (!img) return 0;
        memcpy(img, c->in, sizeof(float) * nxyz);
        memset(c->out, 0, sizeof(float) * nsino);
        if (c->kind == 0)
            ok = cbct_proj_dd(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->ox, c->oy, c->oz, c->nu, c->nv,
                              c->du, c->dv, c->ou, c->ov, c->sad, c->add, c->sdd, c->noviews, betas, couchz,
                              c->detector_type, img, c->out, map);
        else
            ok = cbct_proj_tf(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->ox, c->oy, c->oz, c->nu, c->nv,
                              c->du, c->dv, c->ou, c->ov, c->sad, c->add, c->sdd, c->noviews, betas, couchz,
                              c->detector_type, img, c->out, map);
        free(img);
    } else {
        float *sino = (float *)malloc(sizeof(float) * (nsino > 0 ? nsino : 1));
        if (!sino) return 0;
        memcpy(sino, c->in, sizeof(float) * nsino);
        memset(c->out, 0, sizeof(float) * nxyz);
        switch (c->kind) {
        case 2:
            ok = cbct_back_dd(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->ox, c->oy, c->oz, c->nu, c->nv,
                              c->du, c->dv, c->ou, c->ov, c->sad, c->add, c->sdd, c->noviews, betas, couchz,
                              c->detector_type, c->out, sino, map);
            break;
        case 3:
            ok = cbct_back_tf(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->ox, c->oy, c->oz, c->nu, c->nv,
                              c->du, c->dv, c->ou, c->ov, c->sad, c->add, c->sdd, c->noviews, betas, couchz,
                              c->detector_type, c->out, sino, map);
            break;
        case 4:
        case 5:
            ok = cbct_back_pd(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->ox, c->oy, c->oz, c->nu, c->nv,
                              c->du, c->dv, c->ou, c->ov, c->sad, c->add, c->sdd, c->noviews, betas, couchz,
                              c->detector_type, c->out, sino, map, c->kind == 4);
            break;
        case 6:
            ok = cbct_back_var(c->nx, c->ny, c->nz, c->dx, c->dy, c->dz, c->ox, c->oy, c->oz, c->nu, c->nv,
                               c->du, c->dv, c->ou, c->ov, c->sad, c->add, c->sdd, c->noviews, betas, couchz,
                               c->detector_type, c->out, sino, map, true);
            break;
        default:
            ok = false;
        }
        free(sino);
    }
    return ok ? 1 : 0;
}

/* Single-thread call of one reference projector, exactly as the MEX gateway runs it. */
int ref_cbct_call(int kind, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                  int nu, int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd,
                  int noviews, const double *betas, const float *couchz, int detector_type,
                  const float *in, float *out, const bool *map)
{
    ref_call c = {kind, nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd,
                  noviews, betas, couchz, detector_type, in, out, map};
    return run_one(&c);
}

typedef struct {
    ref_call call;
    int ok;
} ref_job;

static void *job_main(void *arg)
{
    ref_job *j = (ref_job *)arg;
    j->ok = run_one(&j->call);
    return NULL;
}

/*
 * Multi-threaded harness over view chunks (CPU baseline only).  Each thread calls
 * the unmodified reference function on a contiguous slice of views.  Forward
 * projections write disjoint sinogram slices; backprojections each fill a
 * private image that is summed at the end (so the summation order differs from
 * the single-thread reference).
 */
int ref_cbct_call_mt(int nthreads, int kind, int nx, int ny, int nz, float dx, float dy, float dz, float ox,
                     float oy, float oz, int nu, int nv, float du, float dv, float ou, float ov, float sad,
                     float add, float sdd, int noviews, const double *betas, const float *couchz,
                     int detector_type, const float *in, float *out, const bool *map)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > noviews) nthreads = noviews > 0 ? noviews : 1;
    long nxyz = (long)nx * ny * nz;
    long nuv = (long)nu * nv;
    ref_job *jobs = (ref_job *)calloc(nthreads, sizeof(ref_job));
    pthread_t *tids = (pthread_t *)calloc(nthreads, sizeof(pthread_t));
    float *partial = NULL;
    if (!jobs || !tids) return 0;
    if (kind >= 2) {
        partial = (float *)calloc((size_t)nthreads * (nxyz > 0 ? nxyz : 1), sizeof(float));
        if (!partial) return 0;
    }
    int v0 = 0;
    for (int t = 0; t < nthreads; t++) {
        int cnt = noviews / nthreads + (t < noviews % nthreads ? 1 : 0);
        ref_call c = {kind, nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd,
                      cnt, betas + v0, couchz + v0, detector_type, NULL, NULL, map};
        if (kind <= 1) {
            c.in = in;
            c.out = out + (long)v0 * nuv;
        } else {
            c.in = in + (long)v0 * nuv;
            c.out = partial + (long)t * nxyz;
        }
        jobs[t].call = c;
        v0 += cnt;
    }
    for (int t = 0; t < nthreads; t++) pthread_create(&tids[t], NULL, job_main, &jobs[t]);
    int ok = 1;
    for (int t = 0; t < nthreads; t++) {
        pthread_join(tids[t], NULL);
        ok &= jobs[t].ok;
    }
    if (kind >= 2) {
        memset(out, 0, sizeof(float) * nxyz);
        for (int t = 0; t < nthreads; t++) {
            const float *p = partial + (long)t * nxyz;
            for (long i = 0; i < nxyz; i++) out[i] += p[i];
        }
        free(partial);
    }
    free(jobs);
    free(tids);
    return ok;
}
