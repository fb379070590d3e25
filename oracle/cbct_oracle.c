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

#define ORC_FP_DD_U 16 /* iumax <= iumin + 15   geom/cbct/cbct_proj.c:343 */
#define ORC_FP_TF_U 10 /* iumax <= iumin + 9    geom/cbct/cbct_proj.c:612 (FOOTPRINT_SIZE_U = 10, :210) */
#define ORC_FP_V 10    /* ivmax <= ivmin + 9    geom/cbct/cbct_proj.c:395 (FOOTPRINT_SIZE_V = 10, :211) */

enum { ORC_DD = 0, ORC_TF = 1 };

typedef struct {
    int nx, ny, nz, nu, nv, detector_type;
    float dx, dy, dz, sad, sdd, du, dv;
    float wx, wy, wu, wv, sdd_du;
    float oz;
} orc_geom;

/* Per-view constants (geom/cbct/cbct_proj.c:256-265). */
typedef struct {
    float sin_a, cos_a, wz;
    float dx_sin_2, dx_cos_2, dy_sin_2, n_dy_cos_2;
} orc_view;

/* Centre offset "- ( n - 1.0 ) / 2.0 + offset" evaluated in double, stored as float
 * (geom/cbct/cbct_proj.c:244-247). */
static float orc_centre(int n, float offset) { return (float)(-((double)n - 1.0) / 2.0 + (double)offset); }

static orc_geom orc_make_geom(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                              int nu, int nv, float du, float dv, float ou, float ov, float sad, float sdd,
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
    return g;
}

static orc_view orc_make_view(const orc_geom *g, double beta, float couchz)
{
    orc_view v;
    v.sin_a = (float)sin(beta);
    v.cos_a = (float)cos(beta);
    /* wz: geom/cbct/cbct_proj.c:256, the couch shift divided in float then added in double */
    float cz = couchz / g->dz;
    v.wz = (float)((-((double)g->nz - 1.0) / 2.0 + (double)g->oz) + (double)cz);
    /* halves are exact: (x * s) / 2.0   geom/cbct/cbct_proj.c:262-265 */
    v.dx_sin_2 = (float)((double)(g->dx * v.sin_a) / 2.0);
    v.dx_cos_2 = (float)((double)(g->dx * v.cos_a) / 2.0);
    v.dy_sin_2 = (float)((double)(g->dy * v.sin_a) / 2.0);
    v.n_dy_cos_2 = (float)((double)(-g->dy * v.cos_a) / 2.0);
    return v;
}

/* Result of the transaxial (u) footprint of one voxel column in one view. */
typedef struct {
    int hit;           /* 0: the column misses the detector                     */
    int iumin, iumax;  /* detector columns touched                              */
    float w[ORC_FP_DD_U];
    float ampu;        /* in-plane path-length factor dx/max(|cos|,|sin|)/10    */
    float zinc, vstart;/* axial footprint: voxel height in rows, first edge     */
    int iz_start, iz_stop;
} orc_column;

/* Shared column geometry: rotated centre, distance to source, amplitude
 * (geom/cbct/cbct_proj.c:282-310 DD, :531-549 TF). */
static void orc_column_centre(const orc_geom *g, const orc_view *v, int ix, int iy, float *tproj0, float *dsxy0,
                              float *cos_phi, float *sin_phi)
{
    float xc = ((float)ix + g->wx) * g->dx;
    float yc = ((float)iy + g->wy) * g->dy;
    float t = xc * v->cos_a - yc * v->sin_a;
    float d = g->sad + xc * v->sin_a + yc * v->cos_a;
    float r = (float)sqrt((double)(t * t + d * d));
    float cg = d / r;
    float sg = t / r;
    *tproj0 = t;
    *dsxy0 = d;
    *cos_phi = (float)fabs((double)(v->cos_a * cg - v->sin_a * sg));
    *sin_phi = (float)fabs((double)(v->sin_a * cg + v->cos_a * sg));
}

/* Detector coordinate (in pixels, before the +0.5 shift) of the ray through (t, d). */
static float orc_u_of(const orc_geom *g, float num, float den)
{
    if (g->detector_type == 1) return g->sdd_du * num / den - g->wu;
    /* curved: sdd_du * atan(ratio) - wu in double, geom/cbct/cbct_proj.c:316 */
    return (float)((double)g->sdd_du * atan((double)(num / den)) - (double)g->wu);
}

/* Axial part shared by DD and TF (geom/cbct/cbct_proj.c:361-372). */
static int orc_column_axial(const orc_geom *g, const orc_view *v, float dsxy0, orc_column *c)
{
    c->zinc = g->dz / g->dv * g->sdd / dsxy0;
    c->vstart = (float)(((double)v->wz - 0.5) * (double)c->zinc - (double)g->wv);
    int s = (int)floorf((-1.0f - c->vstart) / c->zinc);
    int e = (int)ceilf(((float)(g->nv + 1) - c->vstart) / c->zinc);
    if (s < 0) s = 0;
    if (e > g->nz) e = g->nz;
    c->iz_start = s;
    c->iz_stop = e;
    return s <= e;
}

/* Distance-driven u footprint (geom/cbct/cbct_proj.c:297-359). */
static void orc_column_dd(const orc_geom *g, const orc_view *v, int ix, int iy, orc_column *c)
{
    float tproj0, dsxy0, cos_phi, sin_phi, umin, umax;
    orc_column_centre(g, v, ix, iy, &tproj0, &dsxy0, &cos_phi, &sin_phi);
    c->hit = 0;
    if (cos_phi > sin_phi) {
        c->ampu = (float)((double)(g->dx / cos_phi) / 10.0);
        umin = orc_u_of(g, tproj0 + v->dx_cos_2, dsxy0 + v->dx_sin_2);
        umax = orc_u_of(g, tproj0 - v->dx_cos_2, dsxy0 - v->dx_sin_2);
    } else {
        c->ampu = (float)((double)(g->dx / sin_phi) / 10.0);
        umin = orc_u_of(g, tproj0 + v->dy_sin_2, dsxy0 + v->n_dy_cos_2);
        umax = orc_u_of(g, tproj0 - v->dy_sin_2, dsxy0 - v->n_dy_cos_2);
    }
    if (umin >= umax) { float t = umax; umax = umin; umin = t; }
    umin = umin + 0.5f; if (!(umin > 0.0f)) umin = 0.0f;
    umax = umax + 0.5f; if (!(umax < (float)g->nu)) umax = (float)g->nu;
    if (umin > umax) return;
    int lo = (int)floorf(umin), hi = (int)floorf(umax);
    if (hi > g->nu - 1) hi = g->nu - 1;
    if (hi > lo + ORC_FP_DD_U - 1) hi = lo + ORC_FP_DD_U - 1;
    c->iumin = lo;
    c->iumax = hi;
    if (lo == hi) {
        c->w[0] = umax - umin;
    } else {
        c->w[0] = (float)(lo + 1) - umin;
        for (int k = 1; k < hi - lo; k++) c->w[k] = 1.0f;
        c->w[hi - lo] = umax - (float)hi;
    }
    if (orc_column_axial(g, v, dsxy0, c)) c->hit = 1;
}

/* Separable-footprint (trapezoid) u footprint (geom/cbct/cbct_proj.c:545-643). */
static void orc_column_tf(const orc_geom *g, const orc_view *v, int ix, int iy, orc_column *c)
{
    float tproj0, dsxy0, cos_phi, sin_phi, tau[4];
    orc_column_centre(g, v, ix, iy, &tproj0, &dsxy0, &cos_phi, &sin_phi);
    c->hit = 0;
    c->ampu = (float)((double)(g->dx / (cos_phi > sin_phi ? cos_phi : sin_phi)) / 10.0);
    /* the four corner projections, in the reference's operand order */
    tau[0] = orc_u_of(g, tproj0 + v->dx_cos_2 + v->dy_sin_2, dsxy0 + v->dx_sin_2 + v->n_dy_cos_2);
    tau[1] = orc_u_of(g, tproj0 - v->dx_cos_2 + v->dy_sin_2, dsxy0 - v->dx_sin_2 + v->n_dy_cos_2);
    tau[2] = orc_u_of(g, tproj0 + v->dx_cos_2 - v->dy_sin_2, dsxy0 + v->dx_sin_2 - v->n_dy_cos_2);
    tau[3] = orc_u_of(g, tproj0 - v->dx_cos_2 - v->dy_sin_2, dsxy0 - v->dx_sin_2 - v->n_dy_cos_2);
    /* 5-comparator sorting network: (0,1) (2,3) (0,2) (1,3) (1,2) */
    static const int net[5][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {1, 2}};
    for (int k = 0; k < 5; k++) {
        int a = net[k][0], b = net[k][1];
        if (tau[a] > tau[b]) { float t = tau[a]; tau[a] = tau[b]; tau[b] = t; }
    }
    float umin = tau[0] + 0.5f; if (!(umin > 0.0f)) umin = 0.0f;
    float umax = tau[3] + 0.5f; if (!(umax < (float)g->nu)) umax = (float)g->nu;
    if (umin > umax) return;
    int lo = (int)floorf(umin), hi = (int)floorf(umax);
    if (hi > g->nu - 1) hi = g->nu - 1;
    if (hi > lo + ORC_FP_TF_U - 1) hi = lo + ORC_FP_TF_U - 1;
    c->iumin = lo;
    c->iumax = hi;
    for (int iu = lo; iu <= hi; iu++) {
        float w = 0.0f;
        float bl = (float)((double)iu - 0.5), br = (float)((double)iu + 0.5);
        float xl = bl > tau[0] ? bl : tau[0], xr = br < tau[1] ? br : tau[1];
        if (xr > xl) w = w + (((xr - tau[0]) * (xr - tau[0]) - (xl - tau[0]) * (xl - tau[0])) / (tau[1] - tau[0])) / 2.0f;
        xl = bl > tau[1] ? bl : tau[1]; xr = br < tau[2] ? br : tau[2];
        if (xr > xl) w = w + (xr - xl);
        xl = bl > tau[2] ? bl : tau[2]; xr = br < tau[3] ? br : tau[3];
        if (xr > xl) w = w + (((xl - tau[3]) * (xl - tau[3]) - (xr - tau[3]) * (xr - tau[3])) / (tau[3] - tau[2])) / 2.0f;
        c->w[iu - lo] = w;
    }
    if (orc_column_axial(g, v, dsxy0, c)) c->hit = 1;
}

/* Axial footprint of voxel iz (geom/cbct/cbct_proj.c:382-411): returns the
 * number of detector rows touched (0 = none) and their weights. */
static int orc_voxel_v(const orc_geom *g, const orc_column *c, int iz, int *ivmin, float *wv)
{
    float vmin = c->vstart + (float)iz * c->zinc;
    float vmax = vmin + c->zinc;
    vmin = vmin + 0.5f; if (!(vmin > 0.0f)) vmin = 0.0f;
    vmax = vmax + 0.5f; if (!(vmax < (float)g->nv)) vmax = (float)g->nv;
    if (vmin > vmax) return 0;
    int lo = (int)floorf(vmin), hi = (int)floorf(vmax);
    if (hi > g->nv - 1) hi = g->nv - 1;
    if (hi > lo + ORC_FP_V - 1) hi = lo + ORC_FP_V - 1;
    *ivmin = lo;
    if (lo == hi) {
        wv[0] = vmax - vmin;
    } else {
        wv[0] = (float)(lo + 1) - vmin;
        for (int k = 1; k < hi - lo; k++) wv[k] = 1.0f;
        wv[hi - lo] = vmax - (float)hi;
    }
    return hi - lo + 1;
}

/* Axial amplitude of detector pixel (iu, iv) (geom/cbct/cbct_proj.c:432-450). */
static float orc_ampv(const orc_geom *g, int iu, int iv)
{
    float u = ((float)iu + g->wu) * g->du;
    float uu = g->sdd * g->sdd + u * u;
    float v = ((float)iv + g->wv) * g->dv;
    if (g->detector_type == 1) return (float)sqrt((double)((uu + v * v) / uu));
    return (float)(sqrt((double)(g->sdd * g->sdd + v * v)) / (double)g->sdd);
}

static void orc_column_eval(int kind, const orc_geom *g, const orc_view *v, int ix, int iy, orc_column *c)
{
    if (kind == ORC_DD) orc_column_dd(g, v, ix, iy, c);
    else orc_column_tf(g, v, ix, iy, c);
}

/* Forward projection A (proj,dd / proj,tf), geom/cbct/cbct_proj.c:217-456, :464-744. */
int orc_proj(int kind, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz, int nu,
             int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd, int noviews,
             const double *betas, const float *couchz, int detector_type, const float *image, float *proj,
             const bool *map)
{
    (void)add;
    orc_geom g = orc_make_geom(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, sdd, detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    memset(proj, 0, sizeof(float) * nuv * noviews);
    for (int ib = 0; ib < noviews; ib++) {
        orc_view v = orc_make_view(&g, betas[ib], couchz[ib]);
        float *pv = proj + nuv * ib;
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                orc_column c;
                orc_column_eval(kind, &g, &v, ix, iy, &c);
                if (!c.hit) continue;
                for (int iz = c.iz_start; iz < c.iz_stop; iz++) {
                    float x = image[iz * nxy + (long)iy * nx + ix];
                    if (x == 0.0f) continue;
                    float voxel = c.ampu * x;
                    float wv[ORC_FP_V];
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
             const double *betas, const float *couchz, int detector_type, const float *proj, float *image,
             const bool *map)
{
    (void)add;
    orc_geom g = orc_make_geom(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, sdd, detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    float *scaled = (float *)malloc(sizeof(float) * (nuv > 0 ? nuv : 1));
    if (!scaled) return 0;
    memset(image, 0, sizeof(float) * nxy * nz);
    for (int ib = 0; ib < noviews; ib++) {
        orc_view v = orc_make_view(&g, betas[ib], couchz[ib]);
        const float *pv = proj + nuv * ib;
        for (int iu = 0; iu < nu; iu++)
            for (int iv = 0; iv < nv; iv++) scaled[(long)iu * nv + iv] = pv[(long)iu * nv + iv] * orc_ampv(&g, iu, iv);
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                orc_column c;
                orc_column_eval(kind, &g, &v, ix, iy, &c);
                if (!c.hit) continue;
                for (int iz = c.iz_start; iz < c.iz_stop; iz++) {
                    float wv[ORC_FP_V];
                    int ivmin = 0;
                    int nrow = orc_voxel_v(&g, &c, iz, &ivmin, wv);
                    if (!nrow) continue;
                    float voxel = 0.0f;
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
                const double *betas, const float *couchz, int detector_type, const float *proj, float *image,
                const bool *map, int off_boundary)
{
    (void)add;
    orc_geom g = orc_make_geom(nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov, sad, sdd, detector_type);
    long nxy = (long)nx * ny, nuv = (long)nu * nv;
    float wz = orc_centre(nz, oz); /* no couch term here: geom/cbct/cbct_back.c:47 */
    memset(image, 0, sizeof(float) * nxy * nz);
    for (int ib = 0; ib < noviews; ib++) {
        float sin_a = (float)sin(betas[ib]);
        float cos_a = (float)cos(betas[ib]);
        int couch = (int)couchz[ib]; /* truncated to int: geom/cbct/cbct_back.c:43,52 */
        const float *pv = proj + nuv * ib;
        for (int iy = 0; iy < ny; iy++) {
            for (int ix = 0; ix < nx; ix++) {
                if (!map[iy * nx + ix]) continue;
                float xc = ((float)ix + g.wx) * dx;
                float yc = ((float)iy + g.wy) * dy;
                float xr = xc * cos_a - yc * sin_a;
                float yr = xc * sin_a + yc * cos_a;
                float w2, w2s, u;
                if (detector_type == 1) {
                    w2 = sdd / (sad + yr);
                    w2s = w2 * w2;
                    u = xr * w2 / du - g.wu;
                } else {
                    float roff = ou * du * sad / sdd;
                    u = (float)(atan((double)((xr - roff) / (sad + yr))) * (double)sdd / (double)du - (double)g.wu);
                    w2s = sdd * sdd / ((sad + yr) * (sad + yr) + (xr - roff) * (xr - roff));
                    w2 = sdd / (sad + yr);
                }
                if ((double)u < 1e-6 || (double)u > (double)nu - 1.0 - 1e-6) continue;
                int iu = (int)floorf(u);
                float wul = u - (float)iu;
                for (int iz = 0; iz < nz; iz++) {
                    float zc = ((float)iz + wz) * dz + (float)couch;
                    float vv = zc * w2 / dv - g.wv;
                    if (off_boundary) {
                        if ((double)vv < 1e-6) continue;
                        if ((double)vv > (double)nv - 1.0 - 1e-6) break;
                    } else {
                        vv = (float)((double)vv > 0.5 ? (double)vv : 0.5);
                        vv = (float)((double)vv < (double)nv - 1.5 ? (double)vv : (double)nv - 1.5);
                    }
                    int iv = (int)floorf(vv);
                    float wvl = vv - (float)iv;
                    const float *p = pv + (long)iu * nv + iv;
                    float s0 = (1.0f - wvl) * p[0] + wvl * p[1];
                    float s1 = (1.0f - wvl) * p[nv] + wvl * p[nv + 1];
                    long idx = iz * nxy + (long)iy * nx + ix;
                    image[idx] = image[idx] + w2s * ((1.0f - wul) * s0 + wul * s1);
                }
            }
        }
    }
    return 1;
}
