// Sinogram pre-processing on the device: the data step in front of the projector path.
//   simulate_counts   sinogram/sim/simulateSimplePoissonData.m:161-190 (monochromatic):
//                     intensity = poissrnd(photons .* exp(-line)) + sqrt(electronicNoise) * randn,
//                     or round(photons .* exp(-line)) without counting noise
//   log_attenuation   sinogram/log/computeSimplePoissonSinogramAttunation.m:14-54:
//                     sino = -log(max(intensity, 10) / I0 [./ flatFieldRatio])
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), one counter stream
// per sinogram element, so a draw depends only on (seed, element) and not on the launch.
// Poisson: Hoermann's transformed rejection with squeeze (PTRS, 1993) for lambda >= 10,
// the multiplication method below; both loops are bounded.
#include <cmath>
#include <cstdint>

#include "../../include/ctsim_b200.h"
#include "kernels.cuh"

using namespace ctsim;

extern ctsim_status ctsim_set_last_error(ctsim_status s, const char *msg);

namespace {

constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;  // Philox multipliers
constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;  // Weyl key increments
constexpr int kPtrsTries = 64;                           // PTRS accepts in ~1.1 tries
constexpr int kMultMax = 1000;                           // lambda < 10: k stays far below

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) {
            k0 += kW0;
            k1 += kW1;
        }
        const uint32_t lo0 = kM0 * c.x, hi0 = __umulhi(kM0, c.x);
        const uint32_t lo1 = kM1 * c.z, hi1 = __umulhi(kM1, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    }
    return c;
}

// Uniforms in (0, 1) of one element: Philox blocks (i_lo, i_hi, j, lane) for j = 0, 1, ...
struct Stream {
    uint32_t i0, i1, k0, k1, lane, j;
    uint4 buf;
    int left;
    __device__ Stream(size_t i, uint64_t seed, uint32_t lane_)
        : i0((uint32_t)i), i1((uint32_t)(i >> 32)), k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), lane(lane_),
          j(0), left(0) {}
    __device__ double next() {
        if (left == 0) {
            buf = philox4x32_10(make_uint4(i0, i1, j++, lane), k0, k1);
            left = 4;
        }
        uint32_t w;
        switch (4 - left) {
        case 0: w = buf.x; break;
        case 1: w = buf.y; break;
        case 2: w = buf.z; break;
        default: w = buf.w; break;
        }
        left--;
        return ((double)w + 0.5) * 0x1p-32;
    }
};

// Poisson(lam); *fallback set when the bounded rejection loop gave up (round(lam) returned).
__device__ double poisson(double lam, Stream &s, bool *fallback) {
    if (!(lam > 0.0)) return 0.0;
    if (lam < 10.0) {
        const double lim = exp(-lam);
        int k = 0;
        double prod = s.next();
        while (prod > lim && k < kMultMax) {
            k++;
            prod *= s.next();
        }
        return (double)k;
    }
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int t = 0; t < kPtrsTries; t++) {
        const double U = s.next() - 0.5;
        const double V = s.next();
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0)) return k;
    }
    *fallback = true;
    return floor(lam + 0.5);
}

__global__ void simulate_counts_kernel(const float *__restrict__ line, size_t n, float photons, float noise_sd,
                                       uint64_t seed, int add_noise, float *__restrict__ counts,
                                       unsigned int *__restrict__ fallbacks) {
    unsigned int fb = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        // photons (double scalar) times single exp(-line): computed in single, as MATLAB does
        const float lam = photons * expf(-line[i]);
        if (!add_noise) {
            counts[i] = roundf(lam);  // intensity = round(effectivePhotons)
            continue;
        }
        Stream s(i, seed, 0);
        bool fallback = false;
        double v = poisson((double)lam, s, &fallback);
        fb += fallback;
        if (noise_sd > 0.0f) {
            Stream g(i, seed, 1);
            const double u1 = g.next(), u2 = g.next();
            v += (double)noise_sd * (sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2));  // Box-Muller
        }
        counts[i] = (float)v;
    }
    if (fallbacks && fb) atomicAdd(fallbacks, fb);
}

__global__ void log_attenuation_kernel(const float *__restrict__ counts, size_t n, float source,
                                       const float *__restrict__ flat, size_t nuv, float *__restrict__ sino) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float r = __fdiv_rn(fmaxf(counts[i], 10.0f), source);  // max(intensity, 10) / sourceIntensity
        if (flat) r = __fdiv_rn(r, flat[i % nuv]);               // ./ spectrum.flatFieldRatio
        sino[i] = -logf(r);
    }
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

extern "C" ctsim_status ctsim_simulate_counts(const float *d_line, size_t n, float photons, float electronic_noise,
                                              uint64_t seed, int add_noise, float *d_counts,
                                              unsigned int *d_fallbacks, void *stream) {
    if (!d_line || !d_counts) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (!(photons >= 0.0f) || !(electronic_noise >= 0.0f))
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "photons and electronic noise must be >= 0");
    if (n == 0) return CTSIM_OK;
    simulate_counts_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        d_line, n, photons, sqrtf(electronic_noise), seed, add_noise, d_counts, d_fallbacks);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" ctsim_status ctsim_log_attenuation(const float *d_counts, size_t n, float source_intensity,
                                              const float *d_flat, size_t nuv, float *d_sino, void *stream) {
    if (!d_counts || !d_sino) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (!(source_intensity > 0.0f)) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "source intensity must be > 0");
    if (d_flat && (nuv == 0 || n % nuv != 0))
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "flat-field size must divide the sinogram size");
    if (n == 0) return CTSIM_OK;
    log_attenuation_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_counts, n, source_intensity, d_flat, nuv,
                                                                          d_sino);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CTSIM_OK : ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
}
