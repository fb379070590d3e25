// OS-PWLS building blocks on the device (statsrecon/pwls/reconPwlsSeSqs.m and the
// penalties it loads):
//   pwls_weights     statsrecon/pwls/computeWeightsPwls.m:8-9
//   residual         d = A_s x - y_s, w_s d and sum(w_s d^2)   reconPwlsSeSqs.m:57-74
//   penalty          penalty/huberPenalty.m:103-160, penalty/quadPenalty.m:296-341
//   sqs_update       x <- max(0, x - (At_s(w d) + beta S(x)) / (precom + beta T(x)))
//                    with S, T gathered inline; NaN/Inf -> 0  reconPwlsSeSqs.m:59-66
//   sqdiff           sum((a - b)^2) for the iteration's rmsd      reconPwlsSeSqs.m:81
//   nesterov_update  the Nesterov step of reconPwlsSeNesterovSqs.m:65-87
// Image layout [nz][ny][nx] (MATLAB x(i,j,k) = img[k][j][i]).  Reductions in FP64.
#include <algorithm>
#include <cmath>

#include "../../include/ctsim_b200.h"
#include "kernels.cuh"

// plan internals (capi.cu)
extern const ctsim_geom *ctsim_plan_geom(const ctsim_plan *p);
extern const float *ctsim_plan_ampv(const ctsim_plan *p);

using namespace ctsim;

extern ctsim_status ctsim_set_last_error(ctsim_status s, const char *msg);

namespace {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ void block_add_double(double v, double *acc) {
    // warp reduce, then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFullMask, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(acc, v);
}

__global__ void weights_kernel(const float *__restrict__ s, float r, float v, float *__restrict__ w, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float si = s[i];
        const float d = si - r;
        const float q = __fdiv_rn(__fmul_rn(d, d), si + v);  // (sino - r).^2 ./ (sino + v)
        w[i] = (si <= r) ? 0.0f : q;                         // w(sino <= r) = 0
    }
}

__global__ void residual_kernel(const float *__restrict__ ax, const void *__restrict__ y,
                                const void *__restrict__ w, int dtype, float w_scale, float *__restrict__ wd,
                                size_t n, double *__restrict__ phi) {
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        // the residual is formed in FP32 whatever the storage type of y and w
        const float d = ax[i] - load_as_float(y, i, dtype);
        const float wi = load_as_float(w, i, dtype) * w_scale;
        wd[i] = wi * d;
        acc += (double)wi * (double)d * (double)d;
    }
    if (phi) block_add_double(acc, phi);
}

// The residual of view_count views written as (w d) * ampv per detector pixel (the
// product A^T forms first, in the same order, so the backprojection of this output equals
// that of the plain residual bit for bit).  Blocks run along the pixels of one view
// (blockIdx.y), so the amplitude index needs no division.
__global__ void residual_scaled_kernel(const float *__restrict__ ax, const void *__restrict__ y,
                                       const void *__restrict__ w, int dtype, float w_scale,
                                       const float *__restrict__ ampv, float *__restrict__ wd, int nuv, int views,
                                       double *__restrict__ phi) {
    double acc = 0.0;
    for (int k = blockIdx.y; k < views; k += gridDim.y) {
        const size_t base = (size_t)k * nuv;
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nuv; p += gridDim.x * blockDim.x) {
            const size_t i = base + p;
            const float d = y ? ax[i] - load_as_float(y, i, dtype) : ax[i];
            const float wi = load_as_float(w, i, dtype) * w_scale;
            wd[i] = (wi * d) * ampv[p];
            acc += (double)wi * (double)d * (double)d;
        }
    }
    if (phi) block_add_double(acc, phi);
}

__global__ void sqdiff_kernel(const float *__restrict__ a, const float *__restrict__ b, size_t n,
                              double *__restrict__ acc_out) {
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double d = (double)a[i] - (double)b[i];
        acc += d * d;
    }
    block_add_double(acc, acc_out);
}

// Neighbour differences of voxel (i, j, k), in the order the MATLAB code applies its
// updates: direction D1 x, D2 y, D3 (x+1, y+1) * axy, D4 (x+1, y-1) * axy, D5 z * az;
// within a direction first the voxel's "+" role, then its "-" role.
struct Nbr {
    float d[10];   // differences
    bool ok[10];   // role exists for this voxel
};

__device__ __forceinline__ Nbr gather_diffs(const float *__restrict__ x, int i, int j, int k, int nx, int ny,
                                            int nz) {
    const size_t nxy = (size_t)nx * ny;
    const size_t c = (size_t)k * nxy + (size_t)j * nx + i;
    const float xc = x[c];
    Nbr n;
    // D1: d = x(i) - x(i+1); + at i (i < nx-1), - at i+1
    n.ok[0] = i < nx - 1; n.d[0] = n.ok[0] ? xc - x[c + 1] : 0.f;
    n.ok[1] = i > 0;      n.d[1] = n.ok[1] ? x[c - 1] - xc : 0.f;
    // D2: along y
    n.ok[2] = j < ny - 1; n.d[2] = n.ok[2] ? xc - x[c + nx] : 0.f;
    n.ok[3] = j > 0;      n.d[3] = n.ok[3] ? x[c - nx] - xc : 0.f;
    // D3: d(a,b) = x(a,b) - x(a+1,b+1); + at (a,b), - at (a+1,b+1)
    n.ok[4] = i < nx - 1 && j < ny - 1; n.d[4] = n.ok[4] ? xc - x[c + nx + 1] : 0.f;
    n.ok[5] = i > 0 && j > 0;           n.d[5] = n.ok[5] ? x[c - nx - 1] - xc : 0.f;
    // D4: d(a,b) = x(a+1,b) - x(a,b+1); + at (a+1,b), - at (a,b+1)
    n.ok[6] = i > 0 && j < ny - 1;      n.d[6] = n.ok[6] ? xc - x[c + nx - 1] : 0.f;
    n.ok[7] = i < nx - 1 && j > 0;      n.d[7] = n.ok[7] ? x[c - nx + 1] - xc : 0.f;
    // D5: along z
    n.ok[8] = k < nz - 1; n.d[8] = n.ok[8] ? xc - x[c + nxy] : 0.f;
    n.ok[9] = k > 0;      n.d[9] = n.ok[9] ? x[c - nxy] - xc : 0.f;
    return n;
}

// Gradient S (mode 1) and curvature T (mode 2) of the penalty at one voxel.
// kind 0 = huber (huberPenalty.m), 1 = quadratic (quadPenalty.m, dQuad(d) = d).
__device__ __forceinline__ void grad_curv(const Nbr &n, int kind, float delta, float axy, float az, float cquad,
                                          float *S, float *T) {
    const float coef[5] = {1.0f, 1.0f, axy, axy, az};
    float s = 0.0f, t = 0.0f;
#pragma unroll
    for (int dir = 0; dir < 5; dir++) {
#pragma unroll
        for (int role = 0; role < 2; role++) {
            const int e = 2 * dir + role;
            if (!n.ok[e]) continue;
            const float d = n.d[e];
            float g, c;
            if (kind == 0) {
                g = d > delta ? delta : (d < -delta ? -delta : d);  // dHuber
                c = fabsf(d) <= delta ? 1.0f : 0.0f;               // cHuber
            } else {
                g = d;
                c = 0.0f;
            }
            const float gc = dir < 2 ? g : __fmul_rn(coef[dir], g);
            s = role == 0 ? __fadd_rn(s, gc) : __fsub_rn(s, gc);
            t = __fadd_rn(t, dir < 2 ? c : __fmul_rn(coef[dir], c));
        }
    }
    *S = s;
    *T = kind == 0 ? t : cquad;
}

// mode 0: value (FP64 accumulation); mode 1: gradient; mode 2: curvature.
__global__ void penalty_kernel(const float *__restrict__ x, float *__restrict__ out, double *__restrict__ value,
                               int kind, int mode, float delta, float axy, float az, float cquad, int nx, int ny,
                               int nz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int k = blockIdx.z;
    double acc = 0.0;
    if (i < nx) {
        const Nbr n = gather_diffs(x, i, j, k, nx, ny, nz);
        if (mode == 0) {
            // each difference counted once, at its "+" voxel (roles 0 of each direction)
            const double c[5] = {1.0, 1.0, (double)axy, (double)axy, (double)az};
            for (int dir = 0; dir < 5; dir++) {
                if (!n.ok[2 * dir]) continue;
                const double a = fabs((double)n.d[2 * dir]);
                double h;
                if (kind == 0) h = a <= delta ? a * a / 2 : (double)delta * a - (double)delta * delta / 2;
                else h = a * a / 2;
                acc += c[dir] * h;
            }
        } else {
            float S, T;
            grad_curv(n, kind, delta, axy, az, cquad, &S, &T);
            out[(size_t)k * nx * ny + (size_t)j * nx + i] = mode == 1 ? S : T;
        }
    }
    if (mode == 0) {
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFullMask, acc, o);
        if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(value, acc);
    }
}

// x_new = x - (num + beta S(x)) / (precom + beta T(x)), then x < 0, NaN, Inf -> 0.
// The surrogate denominator and the step are formed in FP64.
__global__ void sqs_update_kernel(const float *__restrict__ x, float *__restrict__ xn, const float *__restrict__ num,
                                  const float *__restrict__ precom, int kind, float beta, float delta, float axy,
                                  float az, float cquad, int nx, int ny, int nz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int k = blockIdx.z;
    if (i >= nx) return;
    const size_t c = (size_t)k * nx * ny + (size_t)j * nx + i;
    float S = 0.f, T = 0.f;
    if (beta != 0.0f) {
        const Nbr n = gather_diffs(x, i, j, k, nx, ny, nz);
        grad_curv(n, kind, delta, axy, az, cquad, &S, &T);
    }
    const double numer = (double)num[c] + (double)beta * (double)S;
    const double denom = (double)precom[c] + (double)beta * (double)T;
    float v = (float)((double)x[c] - numer / denom);
    if (!(v >= 0.0f) || isinf(v)) v = 0.0f;  // x(x<0)=0; isnan -> 0; isinf -> 0
    xn[c] = v;
}

// One subset step of statsrecon/pwls/reconPwlsSeNesterovSqs.m:65-87 at a voxel:
//   du = (num + beta S(z)) / (precom + beta T(x))        (FP64, like sqs_update)
//   x' = z - du;  s' = s - t du;  z' = (1 - 1/t') x' + (1/t') s'
// with z' formed from the unclamped x' and s' (as the MATLAB code orders it), then
// x', s', z' < 0, NaN, Inf -> 0.  s is updated in place (only its own voxel is read).
__global__ void nesterov_update_kernel(const float *__restrict__ z, const float *__restrict__ x,
                                       float *__restrict__ s, const float *__restrict__ num,
                                       const float *__restrict__ precom, float *__restrict__ xn,
                                       float *__restrict__ zn, int kind, float beta, float delta, float axy,
                                       float az, float cquad, double t, double tn, int nx, int ny, int nz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int k = blockIdx.z;
    if (i >= nx) return;
    const size_t c = (size_t)k * nx * ny + (size_t)j * nx + i;
    float Sz = 0.f, Tx = 0.f;
    if (beta != 0.0f) {
        float unused;
        grad_curv(gather_diffs(z, i, j, k, nx, ny, nz), kind, delta, axy, az, cquad, &Sz, &unused);
        grad_curv(gather_diffs(x, i, j, k, nx, ny, nz), kind, delta, axy, az, cquad, &unused, &Tx);
    }
    const double grad = (double)num[c] + (double)beta * (double)Sz;
    const double denom = (double)precom[c] + (double)beta * (double)Tx;
    const double du = grad / denom;
    const float xv = (float)((double)z[c] - du);
    const float sv = (float)((double)s[c] - t * du);
    const float zv = (float)((1.0 - 1.0 / tn) * (double)xv + (1.0 / tn) * (double)sv);
    auto clean = [](float v) { return (!(v >= 0.0f) || isinf(v)) ? 0.0f : v; };
    xn[c] = clean(xv);
    s[c] = clean(sv);
    zn[c] = clean(zv);
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

extern "C" ctsim_status ctsim_pwls_weights(const float *d_counts, float r, float v, float *d_w, size_t n,
                                           void *stream) {
    if (!d_counts || !d_w) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (n == 0) return CTSIM_OK;
    weights_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_counts, r, v, d_w, n);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_pwls_residual_ex(const float *d_ax, const void *d_y, const void *d_w, int dtype,
                                               float w_scale, float *d_wd, size_t n, double *d_phi, void *stream) {
    if (!d_ax || !d_y || !d_w || !d_wd) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (dtype < kF32 || dtype > kF16) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown storage type");
    if (n == 0) return CTSIM_OK;
    residual_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_ax, d_y, d_w, dtype, w_scale, d_wd, n, d_phi);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_pwls_residual_scaled(const ctsim_plan *plan, const float *d_ax, const void *d_y,
                                                   const void *d_w, int dtype, float w_scale, float *d_wd,
                                                   int view_count, double *d_phi, void *stream) {
    if (!plan || !d_ax || !d_w || !d_wd) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (dtype < kF32 || dtype > kF16) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown storage type");
    const ctsim_geom &G = *ctsim_plan_geom(plan);
    if (view_count < 0 || view_count > G.noviews)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "view_count outside the plan's views");
    if (view_count == 0) return CTSIM_OK;
    const int nuv = G.nu * G.nv;
    const int gx = std::max(1, std::min((nuv + 255) / 256, 148 * 16 / std::min(view_count, 65535)));
    dim3 grid(gx, std::min(view_count, 65535));
    residual_scaled_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(d_ax, d_y, d_w, dtype, w_scale,
                                                                   ctsim_plan_ampv(plan), d_wd, nuv, view_count,
                                                                   d_phi);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_pwls_residual(const float *d_ax, const float *d_y, const float *d_w, float *d_wd,
                                            size_t n, double *d_phi, void *stream) {
    return ctsim_pwls_residual_ex(d_ax, d_y, d_w, kF32, 1.0f, d_wd, n, d_phi, stream);
}

extern "C" ctsim_status ctsim_sqdiff(const float *d_a, const float *d_b, size_t n, double *d_acc, void *stream) {
    if (!d_a || !d_b || !d_acc) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (n == 0) return CTSIM_OK;
    sqdiff_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_a, d_b, n, d_acc);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

static void penalty_consts(float *axy, float *az, float *cquad) {
    const double a = 1.0 / std::sqrt(2.0), b = 0.5;
    *axy = (float)a;
    *az = (float)b;
    *cquad = (float)(4.0 + 4.0 * a + 2.0 * b);  // quadPenalty.m:335
}

extern "C" ctsim_status ctsim_penalty(int kind, int mode, float delta, int nx, int ny, int nz, const float *d_x,
                                      float *d_out, double *d_value, void *stream) {
    if (!d_x || (mode != 0 && !d_out) || (mode == 0 && !d_value) || kind < 0 || kind > 1 || mode < 0 || mode > 2)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "invalid penalty arguments");
    if (nx < 1 || ny < 1 || nz < 1) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "sizes must be positive");
    float axy, az, cq;
    penalty_consts(&axy, &az, &cq);
    dim3 grid((nx + 127) / 128, ny, nz);
    penalty_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(d_x, d_out, d_value, kind, mode, delta, axy, az, cq, nx,
                                                          ny, nz);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_sqs_update(int kind, float beta, float delta, int nx, int ny, int nz, const float *d_x,
                                         float *d_xnew, const float *d_num, const float *d_precom, void *stream) {
    if (!d_x || !d_xnew || !d_num || !d_precom || d_x == d_xnew)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "invalid update arguments (x and x_new must differ)");
    if (kind < 0 || kind > 1) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown penalty");
    float axy, az, cq;
    penalty_consts(&axy, &az, &cq);
    dim3 grid((nx + 127) / 128, ny, nz);
    sqs_update_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(d_x, d_xnew, d_num, d_precom, kind, beta, delta, axy,
                                                             az, cq, nx, ny, nz);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_nesterov_update(int kind, float beta, float delta, int nx, int ny, int nz,
                                              const float *d_z, const float *d_x, float *d_s, const float *d_num,
                                              const float *d_precom, double t, double t_next, float *d_xnew,
                                              float *d_znew, void *stream) {
    if (!d_z || !d_x || !d_s || !d_num || !d_precom || !d_xnew || !d_znew)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    // x_new and z_new must not alias the arrays whose neighbours are read (z, x) or s
    const void *in[3] = {d_z, d_x, d_s};
    for (const void *q : in)
        if (q == d_xnew || q == d_znew)
            return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "x_new and z_new must differ from z, x and s");
    if (d_xnew == d_znew) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "x_new and z_new must differ");
    if (kind < 0 || kind > 1) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown penalty");
    if (nx < 1 || ny < 1 || nz < 1) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "sizes must be positive");
    if (!(t >= 1.0) || !(t_next >= 1.0)) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "momentum t must be >= 1");
    float axy, az, cq;
    penalty_consts(&axy, &az, &cq);
    dim3 grid((nx + 127) / 128, ny, nz);
    nesterov_update_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(d_z, d_x, d_s, d_num, d_precom, d_xnew, d_znew,
                                                                  kind, beta, delta, axy, az, cq, t, t_next, nx, ny,
                                                                  nz);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}
