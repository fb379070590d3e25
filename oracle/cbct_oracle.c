/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load this library; the product path
 * (ctsim_b200) never does.
 *
 * A single-threaded CPU restatement of the reference's cone-beam projectors as
 * Linux runs them (geom/cbct, the C MEX behind cbct_geom_mex).  The arithmetic
 * follows the reference operation by operation so that the result is
 * bit-identical to the compiled reference on x86-64 (no FMA contraction, float
 * temporaries where the reference has float temporaries, double where C
 * promotes to double).  The code structure (footprint helpers, one view loop
 * shared by every projector) is this project's own.
 *
 * Array layouts (geom/cbct/cbct_geom_mex.c:95-118, :218-231):
 *   image[iz*nx*ny + iy*nx + ix]      float, x fastest
 *   proj [ib*nu*nv + iu*nv + iv]      float, v fastest
 *   map  [iy*nx + ix]                 bool
 *
 * Compiled twice (oracle/Makefile): with ORC_REAL=float it is the bit-exact
 * restatement above; with ORC_REAL=double the same control flow runs in double
 * everywhere (sin/cos, footprints, weights, accumulation) -- the FP64 oracle that
 * precision variants are measured against.
 *
 * Deliberate differences from the reference:
 *   - inputs are const: the reference back-projectors scale their sinogram
 *     argument in place (geom/cbct/cbct_back.c:196-214); here a scaled copy of
 *     one view is used instead;
 *   - the distance-driven u footprint keeps up to 16 weights.  The reference
 *     clamps the footprint to 16 bins (geom/cbct/cbct_proj.c:343) but stores the
 *     weights in a 10-entry array (:211, :271), which overflows the stack for
 *     footprints wider than 10 bins; geometries used for parity keep every
 *     footprint at 10 bins or fewer.
 */
#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORC_REAL
#define ORC_REAL float
#endif
typedef ORC_REAL real;  /* float: the bit-exact oracle; double: the FP64 oracle */

#define ORC_FP_DD_U 16 /* iumax <= iumin + 15   geom/cbct/cbct_proj.c:343 */
#define ORC_FP_TF_U 10 /* iumax <= iumin + 9    geom/cbct/cbct_proj.c:612 (FOOTPRINT_SIZE_U = 10, :210) */
#define ORC_FP_V 10    /* ivmax <= ivmin + 9    geom/cbct/cbct_proj.c:395 (FOOTPRINT_SIZE_V = 10, :211) */

enum { ORC_DD = 0, ORC_TF = 1 };

typedef struct {
    int nx, ny, nz, nu, nv, detector_type;
    real dx, dy, dz, sad, sdd, du, dv;
    real wx, wy, wu, wv, sdd_du;
    real oz;
    real add, sad_add; /* arc detector (detector_type 2): radius ADD about the axis, sad/add */
} orc_geom;

/* Per-view constants (geom/cbct/cbct_proj.c:256-265). */
typedef struct {
    real sin_a, cos_a, wz;
    real dx_sin_2, dx_cos_2, dy_sin_2, n_dy_cos_2;
} orc_view;

/* Centre offset "- ( n - 1.0 ) / 2.0 + offset" evaluated in double, stored as float
 * (geom/cbct/cbct_proj.c:244-247). */
static real orc_centre(int n, real offset) { return (real)(-((double)n - 1.0) / 2.0 + (double)offset); }

static orc_geom orc_make_geom(int nx, int ny, int nz, real dx, real dy, real dz, real ox, real oy, real oz,
                              int nu, int nv, real du, real dv, real ou, real ov, real sad, real sdd,
                              int detector_type)
{
    orc_geom g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.nu = nu; g.nv = nv; g.detector_type = detector_type;
    g.dx = dx; g.dy = dy; g.dz = dz; g.sad = sad; g.sdd = sdd; g.du = du; g.dv = dv;
    g.wx = orc_centre(nx, ox);
    g.wy = orc_centre(ny, oy);
    g.wu = orc_centre(nu, ou);
    g.wv = orc_centre(nv, ov);
    g.sdd_du = sdd / du;
    g.oz = oz;
    g.add = 0;
    g.sad_add = 0;
    return g;
}

/* The arc detector needs ADD (geom/cbct/cbct_proj3.c:337-355). */
static orc_geom orc_make_geom_add(int nx, int ny, int nz, real dx, real dy, real dz, real ox, real oy, real oz,
                                  int nu, int nv, real du, real dv, real ou, real ov, real sad, real add, real sdd,
                                  int detector_type)
{
    orc_geom g = orc_make_geom(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, sdd, detector_type);
    g.add = add;
    g.sad_add = sad / add;
    return g;
}

static orc_view orc_make_view(const orc_geom *g, double beta, real couchz)
{
    orc_view v;
    v.sin_a = (real)sin(beta);
    v.cos_a = (real)cos(beta);
    /* wz: geom/cbct/cbct_proj.c:256, the couch shift divided in float then added in double */
    real cz = couchz / g->dz;
    v.wz = (real)((-((double)g->nz - 1.0) / 2.0 + (double)g->oz) + (double)cz);
    /* halves are exact: (x * s) / 2.0   geom/cbct/cbct_proj.c:262-265 */
    v.dx_sin_2 = (real)((double)(g->dx * v.sin_a) / 2.0);
    v.dx_cos_2 = (real)((double)(g->dx * v.cos_a) / 2.0);
    v.dy_sin_2 = (real)((double)(g->dy * v.sin_a) / 2.0);
    v.n_dy_cos_2 = (real)((double)(-g->dy * v.cos_a) / 2.0);
    return v;
}

/* Result of the transaxial (u) footprint of one voxel column in one view. */
typedef struct {
    int hit;           /* 0: the column misses the detector                     */
    int iumin, iumax;  /* detector columns touched                              */
    real w[ORC_FP_DD_U];
    real ampu;        /* in-plane path-length factor dx/max(|cos|,|sin|)/10    */
    real zinc, vstart;/* axial footprint: voxel height in rows, first edge     */
    int iz_start, iz_stop;
} orc_column;

/* Shared column geometry: rotated centre, distance to source, amplitude
 * (geom/cbct/cbct_proj.c:282-310 DD, :531-549 TF). */
static void orc_column_centre(const orc_geom *g, const orc_view *v, int ix, int iy, real *tproj0, real *dsxy0,
                              real *cos_phi, real *sin_phi)
{
    real xc = ((real)ix + g->wx) * g->dx;
    real yc = ((real)iy + g->wy) * g->dy;
    real t = xc * v->cos_a - yc * v->sin_a;
    real d = g->sad + xc * v->sin_a + yc * v->cos_a;
    real r = (real)sqrt((double)(t * t + d * d));
    real cg = d / r;
    real sg = t / r;
    *tproj0 = t;
    *dsxy0 = d;
    *cos_phi = (real)fabs((double)(v->cos_a * cg - v->sin_a * sg));
    *sin_phi = (real)fabs((double)(v->sin_a * cg + v->cos_a * sg));
}

/* Detector coordinate (in pixels, before the +0.5 shift) of the ray through (t, d). */
static real orc_u_of(const orc_geom *g, real num, real den)
{
    if (g->detector_type == 1) return g->sdd_du * num / den - g->wu;
    if (g->detector_type == 2) {
        /* arc: fan angle gam of the ray, arc angle xi = gam + asin(sad/add sin gam) where it
         * meets the arc, u = xi * add / du - wu (geom/cbct/cbct_proj3.c:337-343) */
        real gam = (real)atan((double)(num / den));
        real xi = (real)((double)gam + asin((double)g->sad_add * sin((double)gam)));
        return xi * g->add / g->du - g->wu;
    }
    /* curved: sdd_du * atan(ratio) - wu in double, geom/cbct/cbct_proj.c:316 */
    return (real)((double)g->sdd_du * atan((double)(num / den)) - (double)g->wu);
}

/* Axial part shared by DD and TF (geom/cbct/cbct_proj.c:361-372). */
static int orc_column_axial(const orc_geom *g, const orc_view *v, real dsxy0, orc_column *c)
{
    c->zinc = g->dz / g->dv * g->sdd / dsxy0;
    c->vstart = (real)(((double)v->wz - 0.5) * (double)c->zinc - (double)g->wv);
    int s = (int)floor(((real)-1.0 - c->vstart) / c->zinc);
    int e = (int)ceil(((real)(g->nv + 1) - c->vstart) / c->zinc);
    if (s < 0) s = 0;
    if (e > g->nz) e = g->nz;
    c->iz_start = s;
    c->iz_stop = e;
    return s <= e;
}

/* Distance-driven u footprint (geom/cbct/cbct_proj.c:297-359). */
static void orc_column_dd(const orc_geom *g, const orc_view *v, int ix, int iy, orc_column *c)
{
    real tproj0, dsxy0, cos_phi, sin_phi, umin, umax;
    orc_column_centre(g, v, ix, iy, &tproj0, &dsxy0, &cos_phi, &sin_phi);
    c->hit = 0;
    if (cos_phi > sin_phi) {
        c->ampu = (real)((double)(g->dx / cos_phi) / 10.0);
        umin = orc_u_of(g, tproj0 + v->dx_cos_2, dsxy0 + v->dx_sin_2);
        umax = orc_u_of(g, tproj0 - v->dx_cos_2, dsxy0 - v->dx_sin_2);
    } else {
        c->ampu = (real)((double)(g->dx / sin_phi) / 10.0);
        umin = orc_u_of(g, tproj0 + v->dy_sin_2, dsxy0 + v->n_dy_cos_2);
        if (g->detector_type == 2) /* the arc code takes this edge from the x offsets, cbct_proj3.c:352 */
            umax = orc_u_of(g, tproj0 - v->dx_cos_2, dsxy0 - v->dx_sin_2);
        else
            umax = orc_u_of(g, tproj0 - v->dy_sin_2, dsxy0 - v->n_dy_cos_2);
    }
    if (umin >= umax) { real t = umax; umax = umin; umin = t; }
    umin = umin + (real)0.5; if (!(umin > (real)0.0)) umin = (real)0.0;
    umax = umax + (real)0.5; if (!(umax < (real)g->nu)) umax = (real)g->nu;
    if (umin > umax) return;
    int lo = (int)floor(umin), hi = (int)floor(umax);
    if (hi > g->nu - 1) hi = g->nu - 1;
    if (hi > lo + ORC_FP_DD_U - 1) hi = lo + ORC_FP_DD_U - 1;
    c->iumin = lo;
    c->iumax = hi;
    if (lo == hi) {
        c->w[0] = umax - umin;
    } else {
        c->w[0] = (real)(lo + 1) - umin;
        for (int k = 1; k < hi - lo; k++) c->w[k] = (real)1.0;
        c->w[hi - lo] = umax - (real)hi;
    }
    if (orc_column_axial(g, v, dsxy0, c)) c->hit = 1;
}

/* Separable-footprint (trapezoid) u footprint (geom/cbct/cbct_proj.c:545-643). */
static void orc_column_tf(const orc_geom *g, const orc_view *v, int ix, int iy, orc_column *c)
{
    real tproj0, dsxy0, cos_phi, sin_phi, tau[4];
    orc_column_centre(g, v, ix, iy, &tproj0, &dsxy0, &cos_phi, &sin_phi);
    c->hit = 0;
    c->ampu = (real)((double)(g->dx / (cos_phi > sin_phi ? cos_phi : sin_phi)) / 10.0);
    /* the four corner projections, in the reference's operand order */
    tau[0] = orc_u_of(g, tproj0 + v->dx_cos_2 + v->dy_sin_2, dsxy0 + v->dx_sin_2 + v->n_dy_cos_2);
    tau[1] = orc_u_of(g, tproj0 - v->dx_cos_2 + v->dy_sin_2, dsxy0 - v->dx_sin_2 + v->n_dy_cos_2);
    tau[2] = orc_u_of(g, tproj0 + v->dx_cos_2 - v->dy_sin_2, dsxy0 + v->dx_sin_2 - v->n_dy_cos_2);
    tau[3] = orc_u_of(g, tproj0 - v->dx_cos_2 - v->dy_sin_2, dsxy0 - v->dx_sin_2 - v->n_dy_cos_2);
    /* 5-comparator sorting network: (0,1) (2,3) (0,2) (1,3) (1,2) */
    static const int net[5][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {1, 2}};
    for (int k = 0; k < 5; k++) {
        int a = net[k][0], b = net[k][1];
        if (tau[a] > tau[b]) { real t = tau[a]; tau[a] = tau[b]; tau[b] = t; }
    }
    real umin = tau[0] + (real)0.5; if (!(umin > (real)0.0)) umin = (real)0.0;
    real umax = tau[3] + (real)0.5; if (!(umax < (real)g->nu)) umax = (real)g->nu;
    if (umin > umax) return;
    int lo = (int)floor(umin), hi = (int)floor(umax);
    if (hi > g->nu - 1) hi = g->nu - 1;
    if (hi > lo + ORC_FP_TF_U - 1) hi = lo + ORC_FP_TF_U - 1;
    c->iumin = lo;
    c->iumax = hi;
    for (int iu = lo; iu <= hi; iu++) {
        real w = (real)0.0;
        real bl = (real)((double)iu - 0.5), br = (real)((double)iu + 0.5);
        real xl = bl > tau[0] ? bl : tau[0], xr = br < tau[1] ? br : tau[1];
        if (xr > xl) w = w + (((xr - tau[0]) * (xr - tau[0]) - (xl - tau[0]) * (xl - tau[0])) / (tau[1] - tau[0])) / (real)2.0;
        xl = bl > tau[1] ? bl : tau[1]; xr = br < tau[2] ? br : tau[2];
        if (xr > xl) w = w + (xr - xl);
        xl = bl > tau[2] ? bl : tau[2]; xr = br < tau[3] ? br : tau[3];
        if (xr > xl) w = w + (((xl - tau[3]) * (xl - tau[3]) - (xr - tau[3]) * (xr - tau[3])) / (tau[3] - tau[2])) / (real)2.0;
        c->w[iu - lo] = w;
    }
    if (orc_column_axial(g, v, dsxy0, c)) c->hit = 1;
}

/* Axial footprint of voxel iz (geom/cbct/cbct_proj.c:382-411): returns the
 * number of detector rows touched (0 = none) and their weights. */
static int orc_voxel_v(const orc_geom *g, const orc_column *c, int iz, int *ivmin, real *wv)
{
    real vmin = c->vstart + (real)iz * c->zinc;
    real vmax = vmin + c->zinc;
    vmin = vmin + (real)0.5; if (!(vmin > (real)0.0)) vmin = (real)0.0;
    vmax = vmax + (real)0.5; if (!(vmax < (real)g->nv)) vmax = (real)g->nv;
    if (vmin > vmax) return 0;
    int lo = (int)floor(vmin), hi = (int)floor(vmax);
    if (hi > g->nv - 1) hi = g->nv - 1;
    if (hi > lo + ORC_FP_V - 1) hi = lo + ORC_FP_V - 1;
    *ivmin = lo;
    if (lo == hi) {
        wv[0] = vmax - vmin;
    } else {
        wv[0] = (real)(lo + 1) - vmin;
        for (int k = 1; k < hi - lo; k++) wv[k] = (real)1.0;
        wv[hi - lo] = vmax - (real)hi;
    }
    return hi - lo + 1;
}

/* Axial amplitude of detector pixel (iu, iv) (geom/cbct/cbct_proj.c:432-450). */
static real orc_ampv(const orc_geom *g, int iu, int iv)
{
    real u = ((real)iu + g->wu) * g->du;
    real uu = g->sdd * g->sdd + u * u;
    real v = ((real)iv + g->wv) * g->dv;
    if (g->detector_type == 1) return (real)sqrt((double)((uu + v * v) / uu));
    if (g->detector_type == 2) {
        /* source-to-arc-cell distance squared in double, stored in float (cbct_proj3.c:480-482) */
        double ca = cos((double)(u / g->add)), sa = sin((double)(u / g->add));
        double a = ((double)g->sad + (double)g->add * ca) * ((double)g->sad + (double)g->add * ca) +
                   ((double)g->add * sa) * ((double)g->add * sa);
        real s2 = (real)a;
        return (real)sqrt((double)((s2 + v * v) / s2));
    }
    return (real)(sqrt((double)(g->sdd * g->sdd + v * v)) / (double)g->sdd);
}

static void orc_column_eval(int kind, const orc_geom *g, const orc_view *v, int ix, int iy, orc_column *c)
{
    if (kind == ORC_DD) orc_column_dd(g, v, ix, iy, c);
    else orc_column_tf(g, v, ix, iy, c);
}

/* Forward projection A (proj,dd / proj,tf), geom/cbct/cbct_proj.c:217-456, :464-744. */
int orc_proj(int kind, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz, int nu,
             int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd, int noviews,
             const double *betas, const float *couchz, int detector_type, const real *image, real *proj,
             const bool *map)
{
    /* the arc detector is defined for the distance-driven pair only (cbct_proj3.c, cbct_back3.c) */
    if (detector_type == 2 && kind != ORC_DD) return 0;
    orc_geom g = orc_make_geom_add(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd,
                                   detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    memset(proj, 0, sizeof(real) * nuv * noviews);
    for (int ib = 0; ib < noviews; ib++) {
        orc_view v = orc_make_view(&g, betas[ib], couchz[ib]);
        real *pv = proj + nuv * ib;
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                orc_column c;
                orc_column_eval(kind, &g, &v, ix, iy, &c);
                if (!c.hit) continue;
                for (int iz = c.iz_start; iz < c.iz_stop; iz++) {
                    real x = image[iz * nxy + (long)iy * nx + ix];
                    if (x == (real)0.0) continue;
                    real voxel = c.ampu * x;
                    real wv[ORC_FP_V];
                    int ivmin = 0;
                    int nrow = orc_voxel_v(&g, &c, iz, &ivmin, wv);
                    for (int iu = c.iumin; iu <= c.iumax; iu++)
                        for (int k = 0; k < nrow; k++)
                            pv[(long)iu * nv + ivmin + k] += c.w[iu - c.iumin] * wv[k] * voxel;
                }
            }
        }
        for (int iu = 0; iu < nu; iu++)
            for (int iv = 0; iv < nv; iv++) pv[(long)iu * nv + iv] = pv[(long)iu * nv + iv] * orc_ampv(&g, iu, iv);
    }
    return 1;
}

/* Matched backprojection A^T (back,dd / back,tf), geom/cbct/cbct_back.c:136-372, :375-653. */
int orc_back(int kind, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz, int nu,
             int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd, int noviews,
             const double *betas, const float *couchz, int detector_type, const real *proj, real *image,
             const bool *map)
{
    /* the arc detector is defined for the distance-driven pair only (cbct_proj3.c, cbct_back3.c) */
    if (detector_type == 2 && kind != ORC_DD) return 0;
    orc_geom g = orc_make_geom_add(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, add, sdd,
                                   detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    real *scaled = (real *)malloc(sizeof(real) * (nuv > 0 ? nuv : 1));
    if (!scaled) return 0;
    memset(image, 0, sizeof(real) * nxy * nz);
    for (int ib = 0; ib < noviews; ib++) {
        orc_view v = orc_make_view(&g, betas[ib], couchz[ib]);
        const real *pv = proj + nuv * ib;
        for (int iu = 0; iu < nu; iu++)
            for (int iv = 0; iv < nv; iv++) scaled[(long)iu * nv + iv] = pv[(long)iu * nv + iv] * orc_ampv(&g, iu, iv);
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                orc_column c;
                orc_column_eval(kind, &g, &v, ix, iy, &c);
                if (!c.hit) continue;
                for (int iz = c.iz_start; iz < c.iz_stop; iz++) {
                    real wv[ORC_FP_V];
                    int ivmin = 0;
                    int nrow = orc_voxel_v(&g, &c, iz, &ivmin, wv);
                    if (!nrow) continue;
                    real voxel = (real)0.0;
                    for (int iu = c.iumin; iu <= c.iumax; iu++)
                        for (int k = 0; k < nrow; k++)
                            voxel += scaled[(long)iu * nv + ivmin + k] * c.w[iu - c.iumin] * wv[k];
                    image[iz * nxy + (long)iy * nx + ix] += c.ampu * voxel;
                }
            }
        }
    }
    free(scaled);
    return 1;
}

/* Pixel-driven (voxel-driven bilinear) FDK backprojection, back,pd (off_boundary = 1)
 * and back,hpd (off_boundary = 0): geom/cbct/cbct_back.c:7-133. */
int orc_back_pd(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz, int nu, int nv,
                float du, float dv, float ou, float ov, float sad, float add, float sdd, int noviews,
                const double *betas, const float *couchz, int detector_type, const real *proj, real *image,
                const bool *map, int off_boundary)
{
    (void)add;
    orc_geom g = orc_make_geom(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, sdd, detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    real wz = orc_centre(nz, oz); /* no couch term here: geom/cbct/cbct_back.c:47 */
    memset(image, 0, sizeof(real) * nxy * nz);
    for (int ib = 0; ib < noviews; ib++) {
        real sin_a = (real)sin(betas[ib]);
        real cos_a = (real)cos(betas[ib]);
        int couch = (int)couchz[ib]; /* truncated to int: geom/cbct/cbct_back.c:43,52 */
        const real *pv = proj + nuv * ib;
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                real xc = ((real)ix + g.wx) * dx;
                real yc = ((real)iy + g.wy) * dy;
                real xr = xc * cos_a - yc * sin_a;
                real yr = xc * sin_a + yc * cos_a;
                real w2, w2s, u;
                if (detector_type == 1) {
                    w2 = sdd / (sad + yr);
                    w2s = w2 * w2;
                    u = xr * w2 / du - g.wu;
                } else {
                    real roff = ou * du * sad / sdd;
                    u = (real)(atan((double)((xr - roff) / (sad + yr))) * (double)sdd / (double)du - (double)g.wu);
                    w2s = sdd * sdd / ((sad + yr) * (sad + yr) + (xr - roff) * (xr - roff));
                    w2 = sdd / (sad + yr);
                }
                if ((double)u < 1e-6 || (double)u > (double)nu - 1.0 - 1e-6) continue;
                int iu = (int)floor(u);
                real wul = u - (real)iu;
                for (int iz = 0; iz < nz; iz++) {
                    real zc = ((real)iz + wz) * dz + (real)couch;
                    real vv = zc * w2 / dv - g.wv;
                    if (off_boundary) {
                        if ((double)vv < 1e-6) continue;
                        if ((double)vv > (double)nv - 1.0 - 1e-6) break;
                    } else {
                        vv = (real)((double)vv > 0.5 ? (double)vv : 0.5);
                        vv = (real)((double)vv < (double)nv - 1.5 ? (double)vv : (double)nv - 1.5);
                    }
                    int iv = (int)floor(vv);
                    real wvl = vv - (real)iv;
                    const real *p = pv + (long)iu * nv + iv;
                    real s0 = ((real)1.0 - wvl) * p[0] + wvl * p[1];
                    real s1 = ((real)1.0 - wvl) * p[nv] + wvl * p[nv + 1];
                    long idx = iz * nxy + (long)iy * nx + ix;
                    image[idx] = image[idx] + w2s * (((real)1.0 - wul) * s0 + wul * s1);
                }
            }
        }
    }
    return 1;
}

/* Variance backprojection, back,var: geom/cbct/cbct_back_var.c:1-129 as the MEX calls it
 * (offBoundary = true, geom/cbct/cbct_geom_mex.c:242).  Against back,pd: the couch shift
 * enters wz in voxels (:41) instead of zc in mm, the curved-detector offset is
 * offset_u * sad / sdd (:70, without du), and the weight is w2s^2 (:116). */
int orc_back_var(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz, int nu, int nv,
                 float du, float dv, float ou, float ov, float sad, float add, float sdd, int noviews,
                 const double *betas, const float *couchz, int detector_type, const real *proj, real *image,
                 const bool *map)
{
    (void)add;
    orc_geom g = orc_make_geom(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, sdd, detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    memset(image, 0, sizeof(real) * nxy * nz);
    for (int ib = 0; ib < noviews; ib++) {
        real wz = (real)(-((double)nz - 1.0) / 2.0 + (double)oz + (double)(couchz[ib] / dz));
        real sin_a = (real)sin(betas[ib]);
        real cos_a = (real)cos(betas[ib]);
        const real *pv = proj + nuv * ib;
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                real xc = ((real)ix + g.wx) * dx;
                real yc = ((real)iy + g.wy) * dy;
                real xr = xc * cos_a - yc * sin_a;
                real yr = xc * sin_a + yc * cos_a;
                real w2, w2s, u;
                if (detector_type == 1) {
                    w2 = sdd / (sad + yr);
                    w2s = w2 * w2;
                    u = xr * w2 / du - g.wu;
                } else {
                    real roff = ou * sad / sdd;
                    u = (real)(atan((double)((xr - roff) / (sad + yr))) * (double)sdd / (double)du - (double)g.wu);
                    w2s = sdd * sdd / ((sad + yr) * (sad + yr) + (xr - roff) * (xr - roff));
                    w2 = sdd / (sad + yr);
                }
                if ((double)u < 1e-6 || (double)u > (double)nu - 1.0 - 1e-6) continue;
                int iu = (int)floor(u);
                real wul = u - (real)iu;
                for (int iz = 0; iz < nz; iz++) {
                    real zc = ((real)iz + wz) * dz;
                    real vv = zc * w2 / dv - g.wv;
                    if ((double)vv < 1e-6) continue;
                    if ((double)vv > (double)nv - 1.0 - 1e-6) break;
                    int iv = (int)floor(vv);
                    real wvl = vv - (real)iv;
                    const real *p = pv + (long)iu * nv + iv;
                    real s0 = ((real)1.0 - wvl) * p[0] + wvl * p[1];
                    real s1 = ((real)1.0 - wvl) * p[nv] + wvl * p[nv + 1];
                    long idx = iz * nxy + (long)iy * nx + ix;
                    image[idx] = image[idx] + w2s * w2s * (((real)1.0 - wul) * s0 + wul * s1);
                }
            }
        }
    }
    return 1;
}
