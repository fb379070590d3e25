/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * CPU restatement of the reference's 2-D fan-beam distance-driven and
 * separable-footprint pair (geom/fbct):
 *
 *   fbo_proj(0)  proj,dd   geom/fbct/fbct_proj.c:153-289
 *   fbo_proj(1)  proj,tf   geom/fbct/fbct_proj.c:292-464
 *   fbo_back(0)  back,dd   geom/fbct/fbct_back.c:80-222
 *   fbo_back(1)  back,tf   geom/fbct/fbct_back.c:225-393
 *
 * Image float[ny][nx] (image[iy*nx+ix]), sinogram float[noviews][nu]
 * (proj[ib*nu+iu]); outputs are zero-filled first, as the MEX gateway's
 * mxCreateNumericArray leaves them.  The arithmetic follows the reference's C
 * expression by expression, including the places where a double literal widens
 * a term to double (the first bin of a distance-driven footprint, the +0.5
 * boundary shifts), so the results are bit-identical on x86-64 with
 * -ffp-contract=off.
 */
#include <math.h>
#include <stdbool.h>
#include <string.h>

typedef struct {
    float sin_a, cos_a, dx_sin_2, dx_cos_2, dy_sin_2, n_dy_cos_2;
} fbo_view;

typedef struct {
    int nx, ny, nu, det;
    float dx, dy, sad, sdd, du, wx, wy, wu, sdd_du;
} fbo_geom;

static float fbo_centre(int n, float off) { return (float)(-((double)n - 1.0) / 2.0 + (double)off); }

static fbo_geom fbo_make(int nx, int ny, float dx, float dy, float ox, float oy, int nu, float du, float ou, float sad,
                         float sdd, int det)
{
    fbo_geom g;
    g.nx = nx; g.ny = ny; g.nu = nu; g.det = det;
    g.dx = dx; g.dy = dy; g.sad = sad; g.sdd = sdd; g.du = du;
    g.wx = fbo_centre(nx, ox);
    g.wy = fbo_centre(ny, oy);
    g.wu = fbo_centre(nu, ou);
    g.sdd_du = sdd / du;
    return g;
}

static fbo_view fbo_make_view(const fbo_geom *g, double beta)
{
    fbo_view v;
    v.sin_a = (float)sin(beta);
    v.cos_a = (float)cos(beta);
    v.dx_sin_2 = (float)((double)(g->dx * v.sin_a) / 2.0);
    v.dx_cos_2 = (float)((double)(g->dx * v.cos_a) / 2.0);
    v.dy_sin_2 = (float)((double)(g->dy * v.sin_a) / 2.0);
    v.n_dy_cos_2 = (float)((double)(-g->dy * v.cos_a) / 2.0);
    return v;
}

static float fbo_u(const fbo_geom *g, float num, float den)
{
    if (g->det == 1) return g->sdd_du * num / den - g->wu;
    return (float)((double)g->sdd_du * atan((double)(num / den)) - (double)g->wu);
}

/* Centre, amplitude and the two DD edges (or four SF corners, sorted) of pixel (ix, iy). */
static void fbo_pixel(const fbo_geom *g, const fbo_view *v, int ix, int iy, int tf, float *amp, float *t)
{
    float xc = ((float)ix + g->wx) * g->dx;
    float yc = ((float)iy + g->wy) * g->dy;
    float tp = xc * v->cos_a - yc * v->sin_a;
    float ds = g->sad + xc * v->sin_a + yc * v->cos_a;
    float r = (float)sqrt((double)(tp * tp + ds * ds));
    float cg = ds / r, sg = tp / r;
    float cphi = (float)fabs((double)(v->cos_a * cg - v->sin_a * sg));
    float sphi = (float)fabs((double)(v->sin_a * cg + v->cos_a * sg));
    *amp = (float)((double)(g->dx / (cphi > sphi ? cphi : sphi)) / 10.0);
    if (!tf) {
        if (cphi > sphi) {
            t[0] = fbo_u(g, tp + v->dx_cos_2, ds + v->dx_sin_2);
            t[1] = fbo_u(g, tp - v->dx_cos_2, ds - v->dx_sin_2);
        } else {
            t[0] = fbo_u(g, tp + v->dy_sin_2, ds + v->n_dy_cos_2);
            t[1] = fbo_u(g, tp - v->dy_sin_2, ds - v->n_dy_cos_2);
        }
        if (t[0] >= t[1]) { float s = t[1]; t[1] = t[0]; t[0] = s; }
        return;
    }
    t[0] = fbo_u(g, tp + v->dx_cos_2 + v->dy_sin_2, ds + v->dx_sin_2 + v->n_dy_cos_2);
    t[1] = fbo_u(g, tp - v->dx_cos_2 + v->dy_sin_2, ds - v->dx_sin_2 + v->n_dy_cos_2);
    t[2] = fbo_u(g, tp + v->dx_cos_2 - v->dy_sin_2, ds + v->dx_sin_2 - v->n_dy_cos_2);
    t[3] = fbo_u(g, tp - v->dx_cos_2 - v->dy_sin_2, ds - v->dx_sin_2 - v->n_dy_cos_2);
    static const int net[5][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {1, 2}};
    for (int k = 0; k < 5; k++) {
        int a = net[k][0], b = net[k][1];
        if (t[a] > t[b]) { float s = t[a]; t[a] = t[b]; t[b] = s; }
    }
}

/* Trapezoid area of bin iu (fbct_proj.c:430-456). */
static float fbo_tf_weight(int iu, const float *t)
{
    float w = 0.0f;
    float bl = (float)((double)iu - 0.5), br = (float)((double)iu + 0.5);
    float xl = bl > t[0] ? bl : t[0], xr = br < t[1] ? br : t[1];
    if (xr > xl) w = w + (((xr - t[0]) * (xr - t[0]) - (xl - t[0]) * (xl - t[0])) / (t[1] - t[0])) / 2;
    xl = bl > t[1] ? bl : t[1]; xr = br < t[2] ? br : t[2];
    if (xr > xl) w = w + (xr - xl);
    xl = bl > t[2] ? bl : t[2]; xr = br < t[3] ? br : t[3];
    if (xr > xl) w = w + (((xl - t[3]) * (xl - t[3]) - (xr - t[3]) * (xr - t[3])) / (t[3] - t[2])) / 2;
    return w;
}

/* umin = max(t0 + 0.5, 0), umax = min(t_last + 0.5, nu) in double, stored as float. */
static int fbo_range(const fbo_geom *g, float lo, float hi, float *umin, float *umax, int *iumin, int *iumax)
{
    double a = (double)lo + 0.5, b = (double)hi + 0.5;
    *umin = (float)(a > 0 ? a : 0);
    *umax = (float)(b < g->nu ? b : g->nu);
    if (*umin > *umax) return 0;
    *iumin = (int)floorf(*umin);
    *iumax = (int)floorf(*umax);
    if (*iumax > g->nu - 1) *iumax = g->nu - 1;
    return 1;
}

int fbo_proj(int kind, int nx, int ny, float dx, float dy, float ox, float oy, int nu, float du, float ou, float sad,
             float add, float sdd, int noviews, const double *betas, int det, const float *image, float *proj)
{
    (void)add;
    fbo_geom g = fbo_make(nx, ny, dx, dy, ox, oy, nu, du, ou, sad, sdd, det);
    memset(proj, 0, sizeof(float) * (size_t)nu * noviews);
    for (int ib = 0; ib < noviews; ib++) {
        fbo_view v = fbo_make_view(&g, betas[ib]);
        float *p = proj + (size_t)ib * nu;
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                float amp, t[4], umin, umax;
                int lo, hi;
                fbo_pixel(&g, &v, ix, iy, kind, &amp, t);
                if (!fbo_range(&g, t[0], kind ? t[3] : t[1], &umin, &umax, &lo, &hi)) continue;
                float x = image[iy * nx + ix];
                if (kind == 0) {
                    if (lo == hi) {
                        p[lo] = p[lo] + amp * (umax - umin) * x;
                    } else {
                        for (int iu = lo; iu <= hi; iu++) {
                            if (iu == lo)  /* (iumin + 1.0 - umin) widens the product to double */
                                p[iu] = (float)((double)p[iu] + (double)amp * ((double)lo + 1.0 - (double)umin) * (double)x);
                            else if (iu == hi)
                                p[iu] = p[iu] + amp * (umax - (float)hi) * x;
                            else
                                p[iu] = p[iu] + amp * x;
                        }
                    }
                } else {
                    float voxel = amp * x;
                    for (int iu = lo; iu <= hi; iu++) p[iu] = p[iu] + fbo_tf_weight(iu, t) * voxel;
                }
            }
    }
    return 1;
}

int fbo_back(int kind, int nx, int ny, float dx, float dy, float ox, float oy, int nu, float du, float ou, float sad,
             float add, float sdd, int noviews, const double *betas, int det, const float *proj, float *image)
{
    (void)add;
    fbo_geom g = fbo_make(nx, ny, dx, dy, ox, oy, nu, du, ou, sad, sdd, det);
    memset(image, 0, sizeof(float) * (size_t)nx * ny);
    for (int ib = 0; ib < noviews; ib++) {
        fbo_view v = fbo_make_view(&g, betas[ib]);
        const float *p = proj + (size_t)ib * nu;
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                float amp, t[4];
                fbo_pixel(&g, &v, ix, iy, kind, &amp, t);
                if (kind == 0) {
                    float umin, umax;
                    int lo, hi;
                    if (!fbo_range(&g, t[0], t[1], &umin, &umax, &lo, &hi)) continue;
                    float temp = 0.0f;
                    if (lo == hi) {
                        temp = (umax - umin) * p[lo];
                    } else {
                        for (int iu = lo; iu <= hi; iu++) {
                            if (iu == lo)
                                temp = (float)((double)temp + ((double)lo + 1.0 - (double)umin) * (double)p[iu]);
                            else if (iu == hi)
                                temp = temp + (umax - (float)hi) * p[iu];
                            else
                                temp = temp + p[iu];
                        }
                    }
                    image[iy * nx + ix] = image[iy * nx + ix] + amp * temp;
                } else {
                    /* iumin = max(floorf(t0 + 0.5), 0), iumax = min(ceilf(t3 + 0.5), nu - 1), fbct_back.c:345-346 */
                    int lo = (int)floorf((float)((double)t[0] + 0.5));
                    if (lo < 0) lo = 0;
                    int hi = (int)ceilf((float)((double)t[3] + 0.5));
                    if (hi > nu - 1) hi = nu - 1;
                    if (lo > hi) continue;
                    float temp = 0.0f;
                    for (int iu = lo; iu <= hi; iu++) temp = temp + amp * fbo_tf_weight(iu, t) * p[iu];
                    image[iy * nx + ix] = image[iy * nx + ix] + temp;
                }
            }
    }
    return 1;
}
