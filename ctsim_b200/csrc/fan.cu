// 2-D fan-beam distance-driven and separable-footprint pair (geom/fbct):
//   fan_proj_kernel<TF>   proj,dd  geom/fbct/fbct_proj.c:153-289, proj,tf :292-464
//   fan_back_kernel<TF>   back,dd  geom/fbct/fbct_back.c:80-222,  back,tf :225-393
// Image float[ny][nx], sinogram float[noviews][nu].  Both kernels reproduce the
// reference's float/double operations and its summation order:
// * A is a per-bin gather: one warp per (32 detector bins, view) enumerates the pixels
//   whose footprint can reach its bins row by row (binary search of the monotone
//   projected centre along each row, with a margin), in the reference's (iy, ix)
//   order, and each lane adds the contributions to its bin in that order;
// * A^T is pixel-driven: one thread per pixel runs the views in order.
// No atomics; results do not depend on the launch.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ctsim_b200.h"
#include "kernels.cuh"

using namespace ctsim;

extern ctsim_status ctsim_set_last_error(ctsim_status s, const char *msg);

namespace {

struct FanGeom {
    int nx, ny, nu, det;
    float dx, dy, sad, sdd, du;
    float wx, wy, wu, sdd_du;
    float margin;  // candidate window margin of the forward projector (bins)
};

struct FanView {
    float sin_a, cos_a, dx_sin_2, dx_cos_2, dy_sin_2, n_dy_cos_2;
};

__device__ __forceinline__ float fan_u(const FanGeom &g, float num, float den) {
    if (g.det == 1) return fsub(fdiv(fmul(g.sdd_du, num), den), g.wu);
    return (float)__dsub_rn(__dmul_rn((double)g.sdd_du, atan((double)fdiv(num, den))), (double)g.wu);
}

// Amplitude and the sorted DD edges t[0..1] (or SF corners t[0..3]) of pixel (ix, iy):
// fbct_proj.c:199-246 (DD), :342-404 (SF).
template <bool TF>
__device__ __forceinline__ float fan_pixel(const FanGeom &g, const FanView &v, int ix, int iy, float *t) {
    const float xc = fmul(fadd((float)ix, g.wx), g.dx);
    const float yc = fmul(fadd((float)iy, g.wy), g.dy);
    const float tp = fsub(fmul(xc, v.cos_a), fmul(yc, v.sin_a));
    const float ds = fadd(fadd(g.sad, fmul(xc, v.sin_a)), fmul(yc, v.cos_a));
    const float r = __fsqrt_rn(fadd(fmul(tp, tp), fmul(ds, ds)));
    const float cg = fdiv(ds, r), sg = fdiv(tp, r);
    const float cphi = fabsf(fsub(fmul(v.cos_a, cg), fmul(v.sin_a, sg)));
    const float sphi = fabsf(fadd(fmul(v.sin_a, cg), fmul(v.cos_a, sg)));
    const float amp = fdiv(fdiv(g.dx, cphi > sphi ? cphi : sphi), 10.0f);
    if (!TF) {
        if (cphi > sphi) {
            t[0] = fan_u(g, fadd(tp, v.dx_cos_2), fadd(ds, v.dx_sin_2));
            t[1] = fan_u(g, fsub(tp, v.dx_cos_2), fsub(ds, v.dx_sin_2));
        } else {
            t[0] = fan_u(g, fadd(tp, v.dy_sin_2), fadd(ds, v.n_dy_cos_2));
            t[1] = fan_u(g, fsub(tp, v.dy_sin_2), fsub(ds, v.n_dy_cos_2));
        }
        if (t[0] >= t[1]) { const float s = t[1]; t[1] = t[0]; t[0] = s; }
        return amp;
    }
    t[0] = fan_u(g, fadd(fadd(tp, v.dx_cos_2), v.dy_sin_2), fadd(fadd(ds, v.dx_sin_2), v.n_dy_cos_2));
    t[1] = fan_u(g, fadd(fsub(tp, v.dx_cos_2), v.dy_sin_2), fadd(fsub(ds, v.dx_sin_2), v.n_dy_cos_2));
    t[2] = fan_u(g, fsub(fadd(tp, v.dx_cos_2), v.dy_sin_2), fsub(fadd(ds, v.dx_sin_2), v.n_dy_cos_2));
    t[3] = fan_u(g, fsub(fsub(tp, v.dx_cos_2), v.dy_sin_2), fsub(fsub(ds, v.dx_sin_2), v.n_dy_cos_2));
    float s;
    if (t[0] > t[1]) { s = t[0]; t[0] = t[1]; t[1] = s; }
    if (t[2] > t[3]) { s = t[2]; t[2] = t[3]; t[3] = s; }
    if (t[0] > t[2]) { s = t[0]; t[0] = t[2]; t[2] = s; }
    if (t[1] > t[3]) { s = t[1]; t[1] = t[3]; t[3] = s; }
    if (t[1] > t[2]) { s = t[1]; t[1] = t[2]; t[2] = s; }
    return amp;
}

// Trapezoid area of bin iu (fbct_proj.c:430-456).
__device__ __forceinline__ float fan_tf_weight(int iu, const float *t) {
    float w = 0.0f;
    const float bl = (float)((double)iu - 0.5), br = (float)((double)iu + 0.5);
    float xl = bl > t[0] ? bl : t[0], xr = br < t[1] ? br : t[1];
    if (xr > xl) {
        const float a = fsub(xr, t[0]), b = fsub(xl, t[0]);
        w = fadd(w, fdiv(fdiv(fsub(fmul(a, a), fmul(b, b)), fsub(t[1], t[0])), 2.0f));
    }
    xl = bl > t[1] ? bl : t[1]; xr = br < t[2] ? br : t[2];
    if (xr > xl) w = fadd(w, fsub(xr, xl));
    xl = bl > t[2] ? bl : t[2]; xr = br < t[3] ? br : t[3];
    if (xr > xl) {
        const float a = fsub(xl, t[3]), b = fsub(xr, t[3]);
        w = fadd(w, fdiv(fdiv(fsub(fmul(a, a), fmul(b, b)), fsub(t[3], t[2])), 2.0f));
    }
    return w;
}

// umin = max(lo + 0.5, 0), umax = min(hi + 0.5, nu) (double, stored as float) and the bins.
__device__ __forceinline__ bool fan_range(const FanGeom &g, float lo, float hi, float &umin, float &umax, int &ilo,
                                          int &ihi) {
    const double a = __dadd_rn((double)lo, 0.5), b = __dadd_rn((double)hi, 0.5);
    umin = (float)(a > 0.0 ? a : 0.0);
    umax = (float)(b < (double)g.nu ? b : (double)g.nu);
    if (umin > umax) return false;
    ilo = (int)floorf(umin);
    ihi = min((int)floorf(umax), g.nu - 1);
    return true;
}

constexpr int kFanMaxRows = 4096;

// One warp per (32 bins, view).  Shared memory: per row the first candidate column and
// the running candidate count, then one candidate record per lane.
template <bool TF>
__global__ void __launch_bounds__(32) fan_proj_kernel(FanGeom g, const FanView *__restrict__ views,
                                                      const float *__restrict__ image, float *__restrict__ proj,
                                                      int view_begin, int view_stride) {
    extern __shared__ int fsm[];
    int *row_first = fsm;                      // [ny]
    int *row_off = fsm + g.ny;                 // [ny + 1]
    float *c_t = reinterpret_cast<float *>(row_off + g.ny + 1);  // [4][32]
    float *c_amp = c_t + 4 * 32;               // [32]: DD amplitude, SF amplitude * pixel
    float *c_x = c_amp + 32;                   // [32]: DD pixel value
    int *c_lo = reinterpret_cast<int *>(c_x + 32);
    int *c_hi = c_lo + 32;
    const int lane = threadIdx.x;
    const int iu0 = blockIdx.x * 32;
    const int k = blockIdx.y;
    const FanView v = views[view_begin + k * view_stride];
    const float ulo = (float)iu0 - g.margin, uhi = (float)(iu0 + 32) + g.margin;
    // approximate projected centre (candidate search only; footprints are exact below)
    auto centre = [&](int ix, int iy) {
        const float xc = ((float)ix + g.wx) * g.dx, yc = ((float)iy + g.wy) * g.dy;
        const float r = (xc * v.cos_a - yc * v.sin_a) / (g.sad + xc * v.sin_a + yc * v.cos_a);
        return (g.det == 1 ? g.sdd_du * r : g.sdd_du * atanf(r)) - g.wu + 0.5f;
    };
    for (int iy = lane; iy < g.ny; iy += 32) {
        const bool inc = centre(g.nx - 1, iy) >= centre(0, iy);
        int lo = 0, hi = g.nx;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float f = centre(mid, iy);
            if (inc ? (f < ulo) : (f > uhi)) lo = mid + 1; else hi = mid;
        }
        const int first = lo;
        hi = g.nx;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float f = centre(mid, iy);
            if (inc ? (f > uhi) : (f < ulo)) hi = mid; else lo = mid + 1;
        }
        row_first[iy] = first;
        row_off[iy] = lo - first;
    }
    __syncwarp();
    {   // exclusive scan of the per-row counts (lane owns a contiguous run of rows)
        const int per = (g.ny + 31) / 32;
        const int b = lane * per, e = min(b + per, g.ny);
        int sum = 0;
        for (int iy = b; iy < e; iy++) sum += row_off[iy];
        int incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += n;
        }
        __syncwarp();
        int run = incl - sum;
        for (int iy = b; iy < e; iy++) {
            const int c = row_off[iy];
            row_off[iy] = run;
            run += c;
        }
        if (lane == 31) row_off[g.ny] = incl;
    }
    __syncwarp();
    const int ncand = row_off[g.ny];
    const int iu = iu0 + lane;
    float acc = 0.0f;
    for (int c0 = 0; c0 < ncand; c0 += 32) {
        const int c = c0 + lane;
        int lo = 0, hi = -1;
        if (c < ncand) {
            int a = 0, z = g.ny - 1;  // last row with row_off <= c
            while (a < z) {
                const int mid = (a + z + 1) >> 1;
                if (row_off[mid] <= c) a = mid; else z = mid - 1;
            }
            const int iy = a, ix = row_first[a] + (c - row_off[a]);
            float t[4];
            const float amp = fan_pixel<TF>(g, v, ix, iy, t);
            float umin, umax;
            if (fan_range(g, t[0], TF ? t[3] : t[1], umin, umax, lo, hi)) {
                const float x = image[(size_t)iy * g.nx + ix];
                if (TF) {
                    for (int q = 0; q < 4; q++) c_t[q * 32 + lane] = t[q];
                    c_amp[lane] = fmul(amp, x);  // voxel = amplitude * image
                } else {
                    c_t[lane] = umin;
                    c_t[32 + lane] = umax;
                    c_amp[lane] = amp;
                    c_x[lane] = x;
                }
            } else {
                lo = 0;
                hi = -1;
            }
        }
        c_lo[lane] = lo;
        c_hi[lane] = hi;
        __syncwarp();
        const int ns = min(32, ncand - c0);
        for (int s = 0; s < ns; s++) {
            const int slo = c_lo[s], shi = c_hi[s];
            if (iu < slo || iu > shi) continue;
            if (TF) {
                float t[4] = {c_t[s], c_t[32 + s], c_t[64 + s], c_t[96 + s]};
                acc = fadd(acc, fmul(fan_tf_weight(iu, t), c_amp[s]));
            } else {
                const float umin = c_t[s], umax = c_t[32 + s], amp = c_amp[s], x = c_x[s];
                if (slo == shi) {
                    acc = fadd(acc, fmul(fmul(amp, fsub(umax, umin)), x));
                } else if (iu == slo) {  // amplitude * (iumin + 1.0 - umin) * image, in double
                    const double w = __dsub_rn(__dadd_rn((double)slo, 1.0), (double)umin);
                    acc = (float)__dadd_rn((double)acc, __dmul_rn(__dmul_rn((double)amp, w), (double)x));
                } else if (iu == shi) {
                    acc = fadd(acc, fmul(fmul(amp, fsub(umax, (float)shi)), x));
                } else {
                    acc = fadd(acc, fmul(amp, x));
                }
            }
        }
        __syncwarp();
    }
    if (iu < g.nu) proj[(size_t)k * g.nu + iu] = acc;
}

// One thread per pixel, the views in order (fbct_back.c:114-218 DD, :253-388 SF).
template <bool TF>
__global__ void __launch_bounds__(256) fan_back_kernel(FanGeom g, const FanView *__restrict__ views,
                                                       const float *__restrict__ proj, float *__restrict__ image,
                                                       int view_begin, int view_stride, int view_count, float scale) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y;
    if (ix >= g.nx) return;
    float img = 0.0f;
    for (int k = 0; k < view_count; k++) {
        const FanView v = views[view_begin + k * view_stride];
        const float *p = proj + (size_t)k * g.nu;
        float t[4];
        const float amp = fan_pixel<TF>(g, v, ix, iy, t);
        if (!TF) {
            float umin, umax;
            int lo, hi;
            if (!fan_range(g, t[0], t[1], umin, umax, lo, hi)) continue;
            float temp = 0.0f;
            if (lo == hi) {
                temp = fmul(fsub(umax, umin), __ldg(p + lo));
            } else {
                for (int iu = lo; iu <= hi; iu++) {
                    const float pv = __ldg(p + iu);
                    if (iu == lo) {
                        const double w = __dsub_rn(__dadd_rn((double)lo, 1.0), (double)umin);
                        temp = (float)__dadd_rn((double)temp, __dmul_rn(w, (double)pv));
                    } else if (iu == hi) {
                        temp = fadd(temp, fmul(fsub(umax, (float)hi), pv));
                    } else {
                        temp = fadd(temp, pv);
                    }
                }
            }
            img = fadd(img, fmul(amp, temp));
        } else {
            // iumin = max(floorf(t0 + 0.5), 0), iumax = min(ceilf(t3 + 0.5), nu - 1), fbct_back.c:345-346
            const int lo = max((int)floorf((float)__dadd_rn((double)t[0], 0.5)), 0);
            const int hi = min((int)ceilf((float)__dadd_rn((double)t[3], 0.5)), g.nu - 1);
            if (lo > hi) continue;
            float temp = 0.0f;
            for (int iu = lo; iu <= hi; iu++) temp = fadd(temp, fmul(fmul(amp, fan_tf_weight(iu, t)), __ldg(p + iu)));
            img = fadd(img, temp);
        }
    }
    if (scale != 1.0f) img = img * scale;
    image[(size_t)iy * g.nx + ix] = img;
}

}  // namespace

struct ctsim_fan_plan {
    ctsim_fan_geom geom;
    FanGeom g;
    int device = 0;
    FanView *d_views = nullptr;
};

static size_t fan_proj_smem(int ny) { return (size_t)(2 * ny + 1) * 4 + 32 * 6 * 4 + 32 * 2 * 4; }

extern "C" ctsim_status ctsim_fan_plan_create(const ctsim_fan_geom *geom, const double *betas, ctsim_fan_plan **out) {
    if (!geom || !betas || !out) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    const ctsim_fan_geom G = *geom;
    if (G.nx < 1 || G.ny < 1 || G.nu < 1 || G.noviews < 1)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "sizes must be positive");
    if (!(G.dx > 0 && G.dy > 0 && G.du > 0 && G.sad > 0 && G.sdd > 0))
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "spacings and distances must be positive");
    if (G.detector_type != 0 && G.detector_type != 1)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "detector_type must be 1 (flat) or 0 (curved)");
    if (G.ny > kFanMaxRows) return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "fan-beam images support ny <= 4096");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_NO_DEVICE, cudaGetErrorString(e));
    ctsim_fan_plan *p = new ctsim_fan_plan();
    p->geom = G;
    p->device = dev;
    FanGeom &g = p->g;
    g.nx = G.nx; g.ny = G.ny; g.nu = G.nu; g.det = G.detector_type;
    g.dx = G.dx; g.dy = G.dy; g.sad = G.sad; g.sdd = G.sdd; g.du = G.du;
    g.wx = (float)(-((double)G.nx - 1.0) / 2.0 + (double)G.offset_x);
    g.wy = (float)(-((double)G.ny - 1.0) / 2.0 + (double)G.offset_y);
    g.wu = (float)(-((double)G.nu - 1.0) / 2.0 + (double)G.offset_u);
    g.sdd_du = G.sdd / G.du;
    // margin: half the pixel diagonal magnified at the nearest pixel, stretched at the
    // detector's edge for a flat panel, plus slack for the approximate centre
    double rmax = 0.0;
    for (int cx = 0; cx < 2; cx++)
        for (int cy = 0; cy < 2; cy++) {
            const double xc = ((cx ? G.nx - 1 : 0) + (double)g.wx) * G.dx, yc = ((cy ? G.ny - 1 : 0) + (double)g.wy) * G.dy;
            rmax = std::max(rmax, std::sqrt(xc * xc + yc * yc));
        }
    const double diag = std::sqrt((double)G.dx * G.dx + (double)G.dy * G.dy);
    const double dmin = (double)G.sad - rmax - diag;
    if (!(dmin > 0.0)) {
        delete p;
        return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "the source orbit must lie outside the image (SAD > radius)");
    }
    const double umm = std::max(std::fabs((double)g.wu * G.du), std::fabs(((double)G.nu - 1 + g.wu) * G.du)) + G.du;
    const double stretch = G.detector_type == 1 ? 1.0 + (umm / G.sdd) * (umm / G.sdd) : 1.0;
    g.margin = (float)std::ceil(0.5 * diag * G.sdd / dmin / G.du * stretch) + 2.0f;
    std::vector<FanView> views(G.noviews);
    for (int ib = 0; ib < G.noviews; ib++) {
        FanView &v = views[ib];
        v.sin_a = (float)std::sin(betas[ib]);
        v.cos_a = (float)std::cos(betas[ib]);
        v.dx_sin_2 = (float)((double)(G.dx * v.sin_a) / 2.0);
        v.dx_cos_2 = (float)((double)(G.dx * v.cos_a) / 2.0);
        v.dy_sin_2 = (float)((double)(G.dy * v.sin_a) / 2.0);
        v.n_dy_cos_2 = (float)((double)(-G.dy * v.cos_a) / 2.0);
    }
    if ((e = cudaMalloc(&p->d_views, sizeof(FanView) * G.noviews)) != cudaSuccess ||
        (e = cudaMemcpy(p->d_views, views.data(), sizeof(FanView) * G.noviews, cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(p->d_views);
        delete p;
        return ctsim_set_last_error(CTSIM_ERR_ALLOC, cudaGetErrorString(e));
    }
    *out = p;
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_fan_plan_destroy(ctsim_fan_plan *p) {
    if (p) {
        cudaFree(p->d_views);
        delete p;
    }
    return CTSIM_OK;
}

static ctsim_status fan_views_ok(const ctsim_fan_plan *p, int vb, int vs, int vc) {
    if (vc < 1 || vs < 1 || vb < 0 || (long long)vb + (long long)(vc - 1) * vs >= p->geom.noviews)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "view selection outside the plan's views");
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_fan_project(ctsim_fan_plan *p, int method, const float *d_image, float *d_sino,
                                          int view_begin, int view_stride, int view_count, void *stream) {
    if (!p || !d_image || !d_sino) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (method != CTSIM_PROJ_DD && method != CTSIM_PROJ_TF)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown forward method");
    ctsim_status s = fan_views_ok(p, view_begin, view_stride, view_count);
    if (s != CTSIM_OK) return s;
    const size_t sm = fan_proj_smem(p->g.ny);
    dim3 grid((p->g.nu + 31) / 32, view_count);
    cudaError_t e;
    if (method == CTSIM_PROJ_DD) {
        if ((e = allow_dynamic_smem((const void *)fan_proj_kernel<false>, sm)) != cudaSuccess)
            return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
        fan_proj_kernel<false><<<grid, 32, sm, (cudaStream_t)stream>>>(p->g, p->d_views, d_image, d_sino, view_begin,
                                                                       view_stride);
    } else {
        if ((e = allow_dynamic_smem((const void *)fan_proj_kernel<true>, sm)) != cudaSuccess)
            return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
        fan_proj_kernel<true><<<grid, 32, sm, (cudaStream_t)stream>>>(p->g, p->d_views, d_image, d_sino, view_begin,
                                                                      view_stride);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_fan_backproject(ctsim_fan_plan *p, int method, const float *d_sino, float *d_image,
                                              int view_begin, int view_stride, int view_count, float scale,
                                              void *stream) {
    if (!p || !d_image || !d_sino) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (method != CTSIM_BACK_DD && method != CTSIM_BACK_TF)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown fan-beam backprojection method");
    ctsim_status s = fan_views_ok(p, view_begin, view_stride, view_count);
    if (s != CTSIM_OK) return s;
    dim3 grid((p->g.nx + 127) / 128, p->g.ny);
    if (method == CTSIM_BACK_DD)
        fan_back_kernel<false><<<grid, 128, 0, (cudaStream_t)stream>>>(p->g, p->d_views, d_sino, d_image, view_begin,
                                                                       view_stride, view_count, scale);
    else
        fan_back_kernel<true><<<grid, 128, 0, (cudaStream_t)stream>>>(p->g, p->d_views, d_sino, d_image, view_begin,
                                                                      view_stride, view_count, scale);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

// Host-pointer entry with the reference's fan-beam MEX dispatch (geom/fbct/fbct_geom_mex.c:243-278):
// proj,dd / proj,tf / back,dd / back,tf; synchronous, never exits.
extern "C" bool ctsim_fbct_geom(const char *type, int nx, int ny, float dx, float dy, float offset_x, float offset_y,
                                int nu, float du, float offset_u, float sad, float add, float sdd, int noviews,
                                const double *betas, int detector_type, const float *data, float *out) {
    if (!type || !betas || !data || !out) {
        ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
        return false;
    }
    int method;
    if (!std::strcmp(type, "proj,dd")) method = CTSIM_PROJ_DD;
    else if (!std::strcmp(type, "proj,tf")) method = CTSIM_PROJ_TF;
    else if (!std::strcmp(type, "back,dd")) method = CTSIM_BACK_DD;
    else if (!std::strcmp(type, "back,tf")) method = CTSIM_BACK_TF;
    else {
        ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "unknown or unsupported fan-beam geom type");
        return false;
    }
    const ctsim_fan_geom G = {nx, ny, dx, dy, offset_x, offset_y, nu, du, offset_u, sad, add, sdd, noviews,
                              detector_type};
    ctsim_fan_plan *p = nullptr;
    if (ctsim_fan_plan_create(&G, betas, &p) != CTSIM_OK) return false;
    const bool fwd = method == CTSIM_PROJ_DD || method == CTSIM_PROJ_TF;
    const size_t nimg = (size_t)nx * ny, nsino = (size_t)nu * noviews;
    const size_t nin = fwd ? nimg : nsino, nout = fwd ? nsino : nimg;
    float *din = nullptr, *dout = nullptr;
    bool ok = false;
    cudaError_t e;
    if ((e = cudaMalloc(&din, nin * 4)) == cudaSuccess && (e = cudaMalloc(&dout, nout * 4)) == cudaSuccess &&
        (e = cudaMemcpy(din, data, nin * 4, cudaMemcpyHostToDevice)) == cudaSuccess) {
        const ctsim_status s = fwd ? ctsim_fan_project(p, method, din, dout, 0, 1, noviews, nullptr)
                                   : ctsim_fan_backproject(p, method, din, dout, 0, 1, noviews, 1.0f, nullptr);
        if (s == CTSIM_OK) {
            if ((e = cudaDeviceSynchronize()) == cudaSuccess && (e = cudaMemcpy(out, dout, nout * 4, cudaMemcpyDeviceToHost)) == cudaSuccess)
                ok = true;
            else
                ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
        }
    } else {
        ctsim_set_last_error(CTSIM_ERR_ALLOC, cudaGetErrorString(e));
    }
    cudaFree(din);
    cudaFree(dout);
    ctsim_fan_plan_destroy(p);
    return ok;
}
