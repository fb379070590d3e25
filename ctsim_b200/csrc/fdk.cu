// FDK reconstruction (fbp/reconFDK.m) on the device:
//   1. cosine weight per detector pixel and, for short scans, Parker weight per
//      (view, detector column)                                   reconFDK.m:38-60
//   2. ramp x window filter along every detector row, by FFT with the zero padding
//      of filterFreq.m (length max(64, 2^nextpow2(2 nu - 1)))     reconFDK.m:62-71
//   3. back,hpd backprojection, times dbeta, times 10             reconFDK.m:78-84
// The filter itself is built on the host by the reference's design
// (fbp/filter/designFilter2.m flat, designEquiangularFilter2.m curved).
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ctsim_b200.h"
#include "kernels.cuh"

using namespace ctsim;

extern ctsim_status ctsim_set_last_error(ctsim_status s, const char *msg);
// plan internals shared with capi.cu
extern const double *ctsim_plan_betas(const ctsim_plan *p);
extern const ctsim_geom *ctsim_plan_geom(const ctsim_plan *p);
extern cudaError_t ctsim_plan_alloc(const ctsim_plan *p, void **ptr, size_t n);
extern void ctsim_plan_release(const ctsim_plan *p, void *ptr);
extern cudaError_t ctsim_plan_upload(const ctsim_plan *p, void *dst, const void *src, size_t n);

namespace {

constexpr int kFiltRows = 8;  // detector rows per block (4 complex FFTs)

int fft_order(int nu) {
    // order = max(64, 2^nextpow2(2*len-1)), designFilter2.m:18
    int L = 1;
    while (L < 2 * nu - 1) L <<= 1;
    return L < 64 ? 64 : L;
}

bool window_known(const std::string &w) {
    static const char *names[] = {"ram-lak", "shepp-logan", "cosine", "hamming", "hann", "hann50", "hann75",
                                  "hann80", "B50", "B75", "B80", "C50", "C75", "C80"};
    for (auto n : names)
        if (w == n) return true;
    return false;
}

// |DFT(h)|[0..count) by an iterative radix-2 FFT in double (size a power of two);
// every twiddle is evaluated directly (no recurrence).
std::vector<double> dft_magnitude(const std::vector<double> &h, int count) {
    const int n = (int)h.size();
    int lg = 0;
    while ((1 << lg) < n) lg++;
    std::vector<std::complex<double>> a(n);
    for (int i = 0; i < n; i++) {
        int r = 0;
        for (int b = 0; b < lg; b++) r |= ((i >> b) & 1) << (lg - 1 - b);
        a[r] = h[i];
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int hl = len / 2;
        for (int j = 0; j < hl; j++) {
            const double ang = -2.0 * M_PI * j / len;
            const std::complex<double> w(std::cos(ang), std::sin(ang));
            for (int i = 0; i < n; i += len) {
                const std::complex<double> u = a[i + j], v = a[i + j + hl] * w;
                a[i + j] = u + v;
                a[i + j + hl] = u - v;
            }
        }
    }
    std::vector<double> m(count);
    for (int k = 0; k < count; k++) m[k] = std::sqrt(a[k].real() * a[k].real() + a[k].imag() * a[k].imag());
    return m;
}

// designFilter2.m:18-78 (flat) / designEquiangularFilter2.m:19-78 (curved), in double.
// gamma = du; SDD used by the equiangular kernel.  Returns H[order].
std::vector<double> design_filter(int nu, double du, double sdd, bool flat, const std::string &window, double crop) {
    const int order = fft_order(nu);
    // h over index = -order/2+1 .. order/2-1, then h(order) = 0 (zero padding)
    std::vector<double> h(order, 0.0);
    for (int n = 0; n < order - 1; n++) {
        const int index = -order / 2 + 1 + n;
        if (index == 0) {
            h[n] = 1.0 / (4.0 * du * du);
        } else if (((index % 2) + 2) % 2 == 1) {  // MATLAB mod(index,2)==1 (odd, either sign)
            const double d = flat ? (index * M_PI * du) : (sdd * M_PI * std::sin(index * du / sdd));
            h[n] = -1.0 / (d * d);
        }
    }
    // filt = abs(fft(h)), first order/2+1 bins
    const int half = order / 2 + 1;
    std::vector<double> filt = dft_magnitude(h, half);
    std::string win = window;
    if (win == "hann50" || win == "B50" || win == "C50") crop = 0.5;
    if (win == "hann75" || win == "B75" || win == "C75") crop = 0.75;
    if (win == "hann80" || win == "B80" || win == "C80") crop = 0.80;
    for (int k = 1; k < half; k++) {
        const double w = 2.0 * M_PI * k / order;
        if (win == "shepp-logan") filt[k] *= std::sin(w / (2 * crop)) / (w / (2 * crop));
        else if (win == "cosine" || win == "C50" || win == "C75" || win == "C80") filt[k] *= std::cos(w / (2 * crop));
        else if (win == "hamming") filt[k] *= 0.54 + 0.46 * std::cos(w / crop);
        else if (win == "hann" || win == "hann50" || win == "hann75" || win == "hann80")
            filt[k] *= (1.0 + std::cos(w / crop)) / 2.0;
    }
    for (int k = 0; k < half; k++)
        if (2.0 * M_PI * k / order > M_PI * crop) filt[k] = 0.0;  // crop, designFilter2.m:77
    // symmetric extension [filt ; filt(end-1:-1:2)]
    std::vector<double> H(order);
    for (int k = 0; k < half; k++) H[k] = filt[k];
    for (int k = half; k < order; k++) H[k] = filt[order - k];
    return H;
}

// MATLAB S-function of fbp/weights/shortScanParkerWeight.m:243-252
double parker_s(double b) {
    if (b <= -0.5) return 0.0;
    if (std::fabs(b) < 0.5) return 0.5 * (1.0 + std::sin(M_PI * b));
    return 1.0;
}

// ---------------------------------------------------------------------------
// Row filter: block = (group of 8 detector rows, view).  Rows 2p and 2p+1 are the
// real and imaginary parts of complex signal p (the filter is real and even, so the
// two filtered rows come back as the real and imaginary parts).  Forward FFT:
// radix-2 decimation in time on bit-reversed input; inverse: decimation in
// frequency from natural order, read back bit-reversed.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fdk_filter_kernel(const void *__restrict__ sino, int in_dtype,
                                                         void *__restrict__ out, int out_dtype,
                                                         const float *__restrict__ wcos,
                                                         const float *__restrict__ parker,
                                                         const float *__restrict__ H, const float2 *__restrict__ tw,
                                                         int nu, int nv, int L, int log2L) {
    extern __shared__ float2 buf[];  // [4][L]
    const int k = blockIdx.y;
    const int iv0 = blockIdx.x * kFiltRows;
    const size_t nuv = (size_t)nu * nv;
    const size_t vbase = (size_t)k * nuv;
    const int t = threadIdx.x;
    const int sh = 32 - log2L;
    // load, weight, scatter to bit-reversed positions (zero padding beyond nu)
    for (int i = t; i < L * kFiltRows; i += blockDim.x) {
        const int iu = i >> 3, r = i & 7;
        float x = 0.0f;
        if (iu < nu && iv0 + r < nv) {
            const size_t o = (size_t)iu * nv + iv0 + r;
            x = load_as_float(sino, vbase + o, in_dtype) * wcos[o];  // reconFDK.m:54
            if (parker) x = x * parker[(size_t)k * nu + iu];  // reconFDK.m:66-68
        }
        const int pos = __brev(iu) >> sh;
        float *dst = reinterpret_cast<float *>(buf + (size_t)(r >> 1) * L + pos);
        dst[r & 1] = x;
    }
    __syncthreads();
    const int nb = 4 * (L >> 1);  // butterflies per stage over the 4 signals
    // forward DIT
    for (int s = 0; s < log2L; s++) {
        const int half = 1 << s;
        for (int b = t; b < nb; b += blockDim.x) {
            const int sig = b / (L >> 1), bb = b % (L >> 1);
            const int pos = bb & (half - 1), grp = bb >> s;
            const int i = (grp << (s + 1)) + pos, j = i + half;
            float2 *x = buf + (size_t)sig * L;
            const float2 w = tw[pos << (log2L - 1 - s)];  // exp(-2 pi i pos / (2 half))
            const float2 a = x[i], c = x[j];
            const float2 cw = make_float2(c.x * w.x - c.y * w.y, c.x * w.y + c.y * w.x);
            x[i] = make_float2(a.x + cw.x, a.y + cw.y);
            x[j] = make_float2(a.x - cw.x, a.y - cw.y);
        }
        __syncthreads();
    }
    // multiply by the (real) filter
    for (int i = t; i < 4 * L; i += blockDim.x) {
        const float h = H[i % L];
        float2 v = buf[i];
        buf[i] = make_float2(v.x * h, v.y * h);
    }
    __syncthreads();
    // inverse DIF (twiddles conjugated), natural in, bit-reversed out
    for (int s = log2L - 1; s >= 0; s--) {
        const int half = 1 << s;
        for (int b = t; b < nb; b += blockDim.x) {
            const int sig = b / (L >> 1), bb = b % (L >> 1);
            const int pos = bb & (half - 1), grp = bb >> s;
            const int i = (grp << (s + 1)) + pos, j = i + half;
            float2 *x = buf + (size_t)sig * L;
            const float2 w = tw[pos << (log2L - 1 - s)];
            const float2 a = x[i], c = x[j];
            const float2 d = make_float2(a.x - c.x, a.y - c.y);
            x[i] = make_float2(a.x + c.x, a.y + c.y);
            x[j] = make_float2(d.x * w.x + d.y * w.y, d.y * w.x - d.x * w.y);  // d * conj(w)
        }
        __syncthreads();
    }
    const float inv = 1.0f / (float)L;
    for (int i = t; i < nu * kFiltRows; i += blockDim.x) {
        const int iu = i >> 3, r = i & 7;
        if (iv0 + r >= nv) continue;
        const int pos = __brev(iu) >> sh;
        const float2 v = buf[(size_t)(r >> 1) * L + pos];
        store_from_float(out, vbase + (size_t)iu * nv + iv0 + r, ((r & 1) ? v.y : v.x) * inv, out_dtype);
    }
}

}  // namespace

struct ctsim_fdk {
    ctsim_plan *plan = nullptr;
    int nu = 0, nv = 0, nviews = 0, L = 0, log2L = 0;
    float dbeta = 0.f;
    float *d_H = nullptr, *d_wcos = nullptr, *d_parker = nullptr;
    void *d_filtered = nullptr;  // the filtered sinogram of ctsim_fdk_run_ex, in the input's storage type
    size_t filtered_bytes = 0;
    float2 *d_tw = nullptr;
};

extern "C" ctsim_status ctsim_fdk_design_filter(int nu, float du, float sdd, int detector_type, const char *window,
                                                float crop, double *H, int *order) {
    if (!window || !window_known(window)) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "Invalid window selected.");
    if (nu < 1 || !(du > 0) || !(sdd > 0)) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "invalid detector");
    const int L = fft_order(nu);
    if (order) *order = L;
    if (H) {
        std::vector<double> h = design_filter(nu, du, sdd, detector_type == 1, window, crop);
        std::memcpy(H, h.data(), sizeof(double) * L);
    }
    return CTSIM_OK;
}

// Device memory follows the plan's allocation mode (stream-ordered plans: on the
// plan's stream), so an FDK object is destroyed before its plan.
static void free_fdk(ctsim_fdk *f) {
    if (!f) return;
    ctsim_plan_release(f->plan, f->d_H);
    ctsim_plan_release(f->plan, f->d_wcos);
    ctsim_plan_release(f->plan, f->d_parker);
    ctsim_plan_release(f->plan, f->d_filtered);
    ctsim_plan_release(f->plan, f->d_tw);
    delete f;
}

extern "C" ctsim_status ctsim_fdk_create(ctsim_plan *plan, const char *window, float crop, int short_scan,
                                         ctsim_fdk **out) {
    if (!plan || !out) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (!window || !window_known(window)) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "Invalid window selected.");
    const ctsim_geom &G = *ctsim_plan_geom(plan);
    if (G.detector_type != 0 && G.detector_type != 1)
        return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "FDK needs a flat (1) or curved (0) detector");
    const double *betas = ctsim_plan_betas(plan);
    const bool flat = G.detector_type == 1;
    ctsim_fdk *f = new ctsim_fdk();
    f->plan = plan;
    f->nu = G.nu;
    f->nv = G.nv;
    f->nviews = G.noviews;
    f->L = fft_order(G.nu);
    while ((1 << f->log2L) < f->L) f->log2L++;
    const double SAD = G.sad, SDD = G.sdd, du = G.du, dv = G.dv;
    // detector coordinates u, v in mm (reconFDK.m:33-34)
    std::vector<double> u(G.nu), v(G.nv);
    for (int i = 0; i < G.nu; i++) u[i] = ((-(G.nu - 1) / 2.0 + i) + G.offset_u) * du;
    for (int i = 0; i < G.nv; i++) v[i] = ((-(G.nv - 1) / 2.0 + i) + G.offset_v) * dv;
    // cosine weight (reconFDK.m:39 flat, :44 curved), stored [iu][iv] like the sinogram
    std::vector<float> wcos((size_t)G.nu * G.nv);
    for (int iu = 0; iu < G.nu; iu++)
        for (int iv = 0; iv < G.nv; iv++) {
            double w;
            if (flat) w = SAD * std::sqrt(1.0 + u[iu] * u[iu] / (SDD * SDD)) / std::sqrt(u[iu] * u[iu] + v[iv] * v[iv] + SDD * SDD);
            else w = SAD / SDD * std::cos(u[iu] / std::sqrt(SDD * SDD + v[iv] * v[iv]));
            wcos[(size_t)iu * G.nv + iv] = (float)w;
        }
    std::vector<double> Hd = design_filter(G.nu, du, SDD, flat, window, crop);
    std::vector<float> H(f->L);
    for (int i = 0; i < f->L; i++) H[i] = (float)(du * Hd[i]);  // H = du * designFilter2(...), reconFDK.m:40
    std::vector<float2> tw(f->L / 2);
    for (int i = 0; i < f->L / 2; i++) {
        const double a = -2.0 * M_PI * i / f->L;
        tw[i] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    // Parker short-scan weights (reconFDK.m:41-42, :56-60; shortScanParkerWeight.m)
    std::vector<float> parker;
    double bmin = betas[0], bmax = betas[0];
    for (int k = 0; k < G.noviews; k++) {
        bmin = std::min(bmin, betas[k]);
        bmax = std::max(bmax, betas[k]);
    }
    if (short_scan) {
        const double Tau = flat ? std::fabs(betas[G.noviews - 1] - betas[0]) - M_PI : std::fabs(bmax - bmin) - M_PI;
        parker.resize((size_t)G.noviews * G.nu);
        for (int k = 0; k < G.noviews; k++) {
            const double beta = betas[k] - bmin;
            for (int iu = 0; iu < G.nu; iu++) {
                const double gammas = flat ? std::atan(-u[iu] / SDD) : -u[iu] / SDD;
                const double gamma = -gammas;
                const double w = parker_s(beta / (Tau - 2 * gamma) - 0.5) -
                                 parker_s((beta - M_PI + 2 * gamma) / (Tau + 2 * gamma) - 0.5);
                parker[(size_t)k * G.nu + iu] = (float)w;
            }
        }
    }
    // dbeta (reconFDK.m:78-81)
    double dbeta = G.noviews > 1 ? std::fabs(betas[G.noviews - 1] - betas[0]) / (G.noviews - 1) : 0.0;
    if (!short_scan) dbeta /= 2.0;
    f->dbeta = (float)dbeta;

    cudaError_t e;
    const ctsim_plan *p = plan;
    if ((e = ctsim_plan_alloc(p, (void **)&f->d_H, sizeof(float) * f->L)) != cudaSuccess ||
        (e = ctsim_plan_alloc(p, (void **)&f->d_wcos, sizeof(float) * wcos.size())) != cudaSuccess ||
        (e = ctsim_plan_alloc(p, (void **)&f->d_tw, sizeof(float2) * tw.size())) != cudaSuccess ||
        (short_scan && (e = ctsim_plan_alloc(p, (void **)&f->d_parker, sizeof(float) * parker.size())) != cudaSuccess)) {
        free_fdk(f);
        return ctsim_set_last_error(CTSIM_ERR_ALLOC, cudaGetErrorString(e));
    }
    if ((e = ctsim_plan_upload(p, f->d_H, H.data(), sizeof(float) * f->L)) != cudaSuccess ||
        (e = ctsim_plan_upload(p, f->d_wcos, wcos.data(), sizeof(float) * wcos.size())) != cudaSuccess ||
        (e = ctsim_plan_upload(p, f->d_tw, tw.data(), sizeof(float2) * tw.size())) != cudaSuccess ||
        (short_scan && (e = ctsim_plan_upload(p, f->d_parker, parker.data(), sizeof(float) * parker.size())) != cudaSuccess)) {
        free_fdk(f);
        return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = f;
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_fdk_destroy(ctsim_fdk *f) {
    free_fdk(f);
    return CTSIM_OK;
}

// The row filter of sino (sino_dtype) into out (out_dtype); FP32 arithmetic.
static ctsim_status fdk_filter(ctsim_fdk *f, const void *d_sino, int sino_dtype, void *out, int out_dtype,
                               void *stream) {
    const size_t sm = sizeof(float2) * 4 * f->L;
    if (sm > 200 * 1024) return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "detector too wide for the row filter");
    cudaError_t e = allow_dynamic_smem((const void *)fdk_filter_kernel, sm);
    if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    dim3 grid((f->nv + kFiltRows - 1) / kFiltRows, f->nviews);
    fdk_filter_kernel<<<grid, 256, sm, (cudaStream_t)stream>>>(d_sino, sino_dtype, out, out_dtype, f->d_wcos,
                                                                f->d_parker, f->d_H, f->d_tw, f->nu, f->nv, f->L,
                                                                f->log2L);
    if ((e = cudaGetLastError()) != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_fdk_filter_ex(ctsim_fdk *f, const void *d_sino, int sino_dtype, float *d_filtered,
                                            void *stream) {
    if (!f || !d_sino || !d_filtered) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (sino_dtype < kF32 || sino_dtype > kF16) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown storage type");
    return fdk_filter(f, d_sino, sino_dtype, d_filtered, kF32, stream);
}

extern "C" ctsim_status ctsim_fdk_filter(ctsim_fdk *f, const float *d_sino, float *d_filtered, void *stream) {
    return ctsim_fdk_filter_ex(f, d_sino, kF32, d_filtered, stream);
}

extern "C" ctsim_status ctsim_fdk_run_ex(ctsim_fdk *f, const void *d_sino, int sino_dtype, float *d_image,
                                         void *stream) {
    if (!f || !d_sino || !d_image) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    if (sino_dtype < kF32 || sino_dtype > kF16) return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "unknown storage type");
    // the filtered sinogram is kept in the input's storage type (a BF16/FP16 request holds
    // no FP32 sinogram-sized buffer), allocated at the first run that needs its size
    const size_t need = (size_t)f->nu * f->nv * f->nviews * (sino_dtype == kF32 ? 4 : 2);
    if (f->filtered_bytes < need) {
        ctsim_plan_release(f->plan, f->d_filtered);
        f->d_filtered = nullptr;
        f->filtered_bytes = 0;
        cudaError_t e = ctsim_plan_alloc(f->plan, &f->d_filtered, need);
        if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_ALLOC, cudaGetErrorString(e));
        f->filtered_bytes = need;
    }
    ctsim_status s = fdk_filter(f, d_sino, sino_dtype, f->d_filtered, sino_dtype, stream);
    if (s != CTSIM_OK) return s;
    // img = backProjectMex(sino, geom, 1, 0, 'back,hpd') * dbeta * 10  (reconFDK.m:84)
    s = ctsim_plan_backproject_ex(f->plan, CTSIM_BACK_HPD, f->d_filtered, sino_dtype, d_image, kF32, 0, 1, f->nviews,
                                  f->dbeta, stream);
    if (s != CTSIM_OK) return s;
    const ctsim_geom &G = *ctsim_plan_geom(f->plan);
    cudaError_t e = launch_scale(d_image, (size_t)G.nx * G.ny * G.nz, 10.0f, (cudaStream_t)stream);
    if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_fdk_run(ctsim_fdk *f, const float *d_sino, float *d_image, void *stream) {
    return ctsim_fdk_run_ex(f, d_sino, kF32, d_image, stream);
}

extern "C" float ctsim_fdk_dbeta(const ctsim_fdk *f) { return f ? f->dbeta : 0.0f; }
