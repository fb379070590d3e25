// C ABI: plans (device-resident geometry tables + scratch) and the drop-in
// host-pointer entry points that replace the reference's cbct_*_gpu functions.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ctsim_b200.h"
#include "kernels.cuh"

using namespace ctsim;

namespace {

thread_local std::string g_last_error = "";

ctsim_status fail(ctsim_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

ctsim_status cuda_fail(cudaError_t e, const char *what) {
    return fail(CTSIM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Centre offset "- ( n - 1.0 ) / 2.0 + offset" in double, stored as float
// (geom/cbct/cbct_proj.c:244-247).
float centre(int n, float off) { return (float)(-((double)n - 1.0) / 2.0 + (double)off); }

// Smallest float f with (double)f >= x.
float float_at_or_above(double x) {
    float f = (float)x;
    if ((double)f < x) f = std::nextafter(f, INFINITY);
    return f;
}
// Largest float f with (double)f <= x.
float float_at_or_below(double x) {
    float f = (float)x;
    if ((double)f > x) f = std::nextafter(f, -INFINITY);
    return f;
}

int pow2_at_least(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace

struct ctsim_plan {
    ctsim_geom geom{};
    Geom g{};
    int device = 0;
    View *d_views = nullptr;
    float *d_ampv = nullptr;
    uint8_t *d_map = nullptr;
    float *d_xs = nullptr;   // axial prefix sums [nx*ny][g.xstride] (or pairs [nx*ny][nz+1][2]) -- forward projector scratch
    float *d_ps = nullptr;   // sinogram scaled by ampv [noviews][nu][nv] -- backprojector scratch
    int *d_err = nullptr;
    size_t bytes = 0;
    float margin = 0.f;      // candidate window margin of the forward projector (pixels)
    float zinc_max = 0.f;    // upper bound of a voxel's height in detector rows
    int back_mz = 1, back_qcap = 0, pd_mz = 1;  // A^T (DD) and FDK z-pass depths (tunable)
    int back_mz_tf = 1, back_qcap_tf = 0;       // A^T (SF) z-pass depth (tunable)
    int fwd_groups = 1;      // candidate groups of the forward projector (tunable)
    int fwd_rows = 32;       // row threads per group of the forward projector (tunable)
    bool fwd_pairs = false;  // prefix sums stored as (X, slope) pairs (small volumes; tunable)
    bool fwd_staged = false; // plain sums, candidate columns staged in shared memory (tunable)
    int fwd_slots = 8;       // prefix columns per stage buffer of the staged projector (tunable)
    bool xs_holds_pairs = false;  // the prefix scratch was sized for pairs
    bool fwd_ok = true;
    std::string fwd_reason;
    std::vector<double> betas;  // host copy of the view angles (FDK weights need them)
    // stream-ordered plans allocate from the library pool on this stream and free there
    bool stream_ordered = false;
    cudaStream_t stream = nullptr;
};

// Plan internals for other translation units (fdk.cu).
const double *ctsim_plan_betas(const ctsim_plan *p) { return p->betas.data(); }
const ctsim_geom *ctsim_plan_geom(const ctsim_plan *p) { return &p->geom; }
const float *ctsim_plan_ampv(const ctsim_plan *p) { return p->d_ampv; }

extern "C" const char *ctsim_last_error(void) { return g_last_error.c_str(); }

// Records the calling thread's last-error message for entry points defined in other
// translation units (noalloc.cu).
ctsim_status ctsim_set_last_error(ctsim_status s, const char *msg) { return fail(s, msg); }
extern "C" const char *ctsim_version(void) { return "ctsim_b200 0.1 (sm_100a)"; }

// Library memory pool of a device for stream-ordered plans: memory freed by a
// finished request stays in the pool (release threshold: unlimited) and serves the
// next request's allocations without a device-wide synchronisation.
static cudaError_t library_pool(int dev, cudaMemPool_t *out) {
    static std::mutex m;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(m);
    auto it = pools.find(dev);
    if (it != pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~0ull;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    pools[dev] = pool;
    *out = pool;
    return cudaSuccess;
}

// Allocation, release and upload for a plan and the objects built on it (FDK): the
// runtime's synchronous calls, or stream-ordered ones on the plan's stream.
cudaError_t ctsim_plan_alloc(const ctsim_plan *p, void **ptr, size_t n) {
    if (!p->stream_ordered) return cudaMalloc(ptr, n);
    cudaMemPool_t pool;
    cudaError_t e = library_pool(p->device, &pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(ptr, n, pool, p->stream);
}
void ctsim_plan_release(const ctsim_plan *p, void *ptr) {
    if (!ptr) return;
    if (p->stream_ordered) cudaFreeAsync(ptr, p->stream);
    else cudaFree(ptr);
}
// Host source may be released when this returns (pageable copies are staged).
cudaError_t ctsim_plan_upload(const ctsim_plan *p, void *dst, const void *src, size_t n) {
    if (!p->stream_ordered) return cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice);
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, p->stream);
}

static void free_plan(ctsim_plan *p) {
    if (!p) return;
    ctsim_plan_release(p, p->d_views);
    ctsim_plan_release(p, p->d_ampv);
    ctsim_plan_release(p, p->d_map);
    ctsim_plan_release(p, p->d_xs);
    ctsim_plan_release(p, p->d_ps);
    ctsim_plan_release(p, p->d_err);
    delete p;
}

static ctsim_status create_plan(const ctsim_geom *geom, const double *betas, const float *couchz, const bool *map,
                                bool stream_ordered, cudaStream_t stream, ctsim_plan **out);

// Rows of one A^T z pass of 32*mz voxels (+2 partial rows, +3 for the 4-row alignment),
// rounded to the 128-row passes of the row buffer.
static int back_qcap_for(const ctsim_plan *p, int mz) {
    const int rows = std::min(p->geom.nv, (int)std::ceil(32.0 * mz * p->zinc_max) + 2) + 4;
    return (rows + 127) / 128 * 128;
}
static bool back_mz_fits(const ctsim_plan *p, int mz) { return back_smem_bytes(back_qcap_for(p, mz)) <= 200 * 1024; }

extern "C" ctsim_status ctsim_plan_create(const ctsim_geom *geom, const double *betas, const float *couchz,
                                          const bool *map, ctsim_plan **out) {
    return create_plan(geom, betas, couchz, map, false, nullptr, out);
}

extern "C" ctsim_status ctsim_plan_create_async(const ctsim_geom *geom, const double *betas, const float *couchz,
                                                const bool *map, void *stream, ctsim_plan **out) {
    return create_plan(geom, betas, couchz, map, true, (cudaStream_t)stream, out);
}

extern "C" ctsim_status ctsim_pool_trim(size_t keep_bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    cudaMemPool_t pool;
    if ((e = library_pool(dev, &pool)) != cudaSuccess) return cuda_fail(e, "memory pool");
    if ((e = cudaMemPoolTrimTo(pool, keep_bytes)) != cudaSuccess) return cuda_fail(e, "cudaMemPoolTrimTo");
    return CTSIM_OK;
}

static ctsim_status create_plan(const ctsim_geom *geom, const double *betas, const float *couchz, const bool *map,
                                bool stream_ordered, cudaStream_t stream, ctsim_plan **out) {
    if (!geom || !betas || !couchz || !out) return fail(CTSIM_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    const ctsim_geom G = *geom;
    if (G.nx < 1 || G.ny < 1 || G.nz < 1 || G.nu < 2 || G.nv < 2 || G.noviews < 1)
        return fail(CTSIM_ERR_ARGUMENT, "sizes must be positive (nu, nv >= 2)");
    if (!(G.dx > 0 && G.dy > 0 && G.dz > 0 && G.du > 0 && G.dv > 0 && G.sad > 0 && G.sdd > 0))
        return fail(CTSIM_ERR_ARGUMENT, "spacings and distances must be positive");
    if (G.detector_type != 0 && G.detector_type != 1 && G.detector_type != 2)
        return fail(CTSIM_ERR_ARGUMENT, "detector_type must be 1 (flat), 0 (curved) or 2 (arc)");
    if (G.detector_type == 2 && !(G.add > 0))
        return fail(CTSIM_ERR_ARGUMENT, "the arc detector needs ADD > 0");
    const long long nxy = (long long)G.nx * G.ny;
    if (nxy * G.nz > (1LL << 31) - 1 || (long long)G.nu * G.nv * G.noviews > (1LL << 40))
        return fail(CTSIM_ERR_ARGUMENT, "volume too large");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(CTSIM_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    if (prop.major != 10) return fail(CTSIM_ERR_NO_DEVICE, "ctsim_b200 is built for sm_100a (B200) only");

    ctsim_plan *p = new ctsim_plan();
    p->geom = G;
    p->device = dev;
    p->stream_ordered = stream_ordered;
    p->stream = stream;
    p->betas.assign(betas, betas + G.noviews);
    Geom &g = p->g;
    g.nx = G.nx; g.ny = G.ny; g.nz = G.nz; g.nu = G.nu; g.nv = G.nv; g.det = G.detector_type;
    g.dx = G.dx; g.dy = G.dy; g.dz = G.dz; g.sad = G.sad; g.sdd = G.sdd; g.du = G.du; g.dv = G.dv;
    g.wx = centre(G.nx, G.offset_x);
    g.wy = centre(G.ny, G.offset_y);
    g.wu = centre(G.nu, G.offset_u);
    g.wv = centre(G.nv, G.offset_v);
    g.sdd_du = G.sdd / G.du;
    g.dz_dv = G.dz / G.dv;
    g.wz_pd = centre(G.nz, G.offset_z);
    g.xstride = prefix_stride(G.nz);
    g.roff = G.offset_u * G.du * G.sad / G.sdd;
    g.roff_var = G.offset_u * G.sad / G.sdd;
    g.add = G.add;
    g.sad_add = G.detector_type == 2 ? G.sad / G.add : 0.0f;
    g.u_lo = float_at_or_above(1e-6);
    g.u_hi = float_at_or_below((double)G.nu - 1.0 - 1e-6);
    g.v_lo = float_at_or_above(1e-6);
    g.v_hi = float_at_or_below((double)G.nv - 1.0 - 1e-6);
    g.v_clamp_lo = 0.5f;
    g.v_clamp_hi = (float)((double)G.nv - 1.5);
    {
        // RN(1/dv) (double then float: innocuous double rounding); a significand of all
        // ones is the one case where the reciprocal-based quotient may misround
        int ex;
        const double m = std::frexp((double)G.dv, &ex);
        const bool all_ones = (float)m == (float)(1.0 - std::ldexp(1.0, -24));
        g.rdv = all_ones ? 0.0f : (float)(1.0 / (double)G.dv);
    }

    // per-view table, geom/cbct/cbct_proj.c:256-265, cbct_back.c:47-52
    std::vector<View> views(G.noviews);
    for (int ib = 0; ib < G.noviews; ib++) {
        View &v = views[ib];
        v.sin_a = (float)std::sin(betas[ib]);
        v.cos_a = (float)std::cos(betas[ib]);
        const float cz = couchz[ib] / G.dz;
        v.wz = (float)((-((double)G.nz - 1.0) / 2.0 + (double)G.offset_z) + (double)cz);
        v.dx_sin_2 = (float)((double)(G.dx * v.sin_a) / 2.0);
        v.dx_cos_2 = (float)((double)(G.dx * v.cos_a) / 2.0);
        v.dy_sin_2 = (float)((double)(G.dy * v.sin_a) / 2.0);
        v.n_dy_cos_2 = (float)((double)(-G.dy * v.cos_a) / 2.0);
        v.couch_pd = (float)(int)couchz[ib];
    }
    // axial amplitude per detector pixel, geom/cbct/cbct_proj.c:432-450
    std::vector<float> ampv((size_t)G.nu * G.nv);
    for (int iu = 0; iu < G.nu; iu++) {
        const float u = ((float)iu + g.wu) * G.du;
        const float uu = G.sdd * G.sdd + u * u;
        for (int iv = 0; iv < G.nv; iv++) {
            const float v = ((float)iv + g.wv) * G.dv;
            float a;
            if (G.detector_type == 1) {
                a = (float)std::sqrt((double)((uu + v * v) / uu));
            } else if (G.detector_type == 0) {
                a = (float)(std::sqrt((double)(G.sdd * G.sdd + v * v)) / (double)G.sdd);
            } else {  // arc: squared source-to-cell distance in double, stored in float (cbct_proj3.c:480-482)
                const double ca = std::cos((double)(u / G.add)), sa = std::sin((double)(u / G.add));
                const float s2 = (float)(((double)G.sad + (double)G.add * ca) * ((double)G.sad + (double)G.add * ca) +
                                         ((double)G.add * sa) * ((double)G.add * sa));
                a = (float)std::sqrt((double)((s2 + v * v) / s2));
            }
            ampv[(size_t)iu * G.nv + iv] = a;
        }
    }
    std::vector<uint8_t> mp((size_t)nxy, 1);
    if (map)
        for (long long i = 0; i < nxy; i++) mp[i] = map[i] ? 1 : 0;

    // Bounds used to size the kernels: the largest distance of a voxel column
    // centre from the rotation axis, hence the smallest source distance.
    double rmax = 0.0;
    for (int cx = 0; cx < 2; cx++)
        for (int cy = 0; cy < 2; cy++) {
            const double xc = ((cx ? G.nx - 1 : 0) + (double)g.wx) * G.dx;
            const double yc = ((cy ? G.ny - 1 : 0) + (double)g.wy) * G.dy;
            rmax = std::max(rmax, std::sqrt(xc * xc + yc * yc));
        }
    const double diag = std::sqrt((double)G.dx * G.dx + (double)G.dy * G.dy);
    const double dmin = (double)G.sad - rmax - diag;
    if (!(dmin > 0.0)) {
        free_plan(p);
        return fail(CTSIM_ERR_UNSUPPORTED, "the source orbit must lie outside the volume (SAD > volume radius)");
    }
    p->zinc_max = (float)((double)G.dz / G.dv * G.sdd / ((double)G.sad - rmax) * 1.0001 + 1e-6);
    const double umm = std::max(std::fabs((double)g.wu * G.du), std::fabs(((double)G.nu - 1 + g.wu) * G.du)) + G.du;
    double stretch = G.detector_type == 1 ? 1.0 + (umm / G.sdd) * (umm / G.sdd) : 1.0;
    if (G.detector_type == 2) {
        // arc: du/dgamma = add (1 + k cos g / sqrt(1 - k^2 sin^2 g)), k = sad/add, grows with
        // the fan angle; sdd = sad + add is its value at g = 0
        const double k = (double)G.sad / G.add;
        const double sg = std::min(1.0, (rmax + diag) / G.sad);  // largest |sin(fan angle)| of a voxel edge
        if (k * sg >= 0.999) {
            free_plan(p);
            return fail(CTSIM_ERR_UNSUPPORTED,
                        "arc detector: the volume's fan angle leaves the arc (sad/add * sin(gamma) >= 1)");
        }
        const double cg = std::sqrt(1.0 - sg * sg);
        stretch = (1.0 + k * cg / std::sqrt(1.0 - k * k * sg * sg)) / (1.0 + k) * ((double)G.sad + G.add) / G.sdd;
        stretch = std::max(stretch, 1.0);
    }
    // candidate window of the forward projector: a voxel's u footprint lies within this many
    // pixels of its projected centre (half the voxel diagonal at the largest magnification,
    // times the detector's stretch), plus half a pixel for the float search
    p->margin = (float)(0.5 * diag * G.sdd / dmin / G.du * stretch * 1.0001 + 0.5);
    if (p->zinc_max > 9.0f) {
        // the kernels integrate the axial footprint exactly; the reference truncates
        // footprints wider than 10 rows (cbct_proj.c:395), which they do not reproduce
        p->fwd_ok = false;
        p->fwd_reason = "distance-driven/separable-footprint projectors need every voxel's axial footprint within 10 detector rows (dz/dv*SDD/dist <= 9)";
    }
    if (G.nx > proj_max_lines() || G.ny > proj_max_lines()) {
        p->fwd_ok = false;
        p->fwd_reason = "forward projection supports nx, ny <= 2048";
    }
    p->fwd_groups = proj_default_groups(G.nv);
    p->fwd_rows = proj_default_rows(G.nv);
    if (proj_smem_bytes(G.nv, G.nx, G.ny, p->fwd_groups) > 200 * 1024) {
        p->fwd_ok = false;
        p->fwd_reason = "forward projection supports nv <= 6080";
    }
    // A^T: z pass of 32*MZ voxels and the per-warp row buffer that covers its shadow
    {
        int mz = std::min(8, pow2_at_least((G.nz + 31) / 32));
        while (mz > 1 && !back_mz_fits(p, mz)) mz >>= 1;
        p->back_mz = p->back_mz_tf = mz;
        p->back_qcap = p->back_qcap_tf = back_qcap_for(p, mz);
        // FDK: one z block of 32 voxels per lane measured fastest on B200 (config 2:
        // 124 ms against 179 ms for eight)
        p->pd_mz = 1;
    }

    // device allocations
    size_t bytes = 0;
#define CTSIM_ALLOC(ptr, n)                                                          \
    do {                                                                             \
        e = ctsim_plan_alloc(p, (void **)&(ptr), (n));                               \
        if (e != cudaSuccess) {                                                      \
            free_plan(p);                                                            \
            return fail(CTSIM_ERR_ALLOC, std::string("device allocation: ") + cudaGetErrorString(e)); \
        }                                                                            \
        bytes += (n);                                                                \
    } while (0)
    CTSIM_ALLOC(p->d_views, sizeof(View) * G.noviews);
    CTSIM_ALLOC(p->d_ampv, sizeof(float) * ampv.size());
    CTSIM_ALLOC(p->d_map, mp.size());
    CTSIM_ALLOC(p->d_err, sizeof(int));
    p->fwd_pairs = p->xs_holds_pairs = forward_pairs(nxy, G.nz);
    // volumes whose prefix sums do not stay cache-resident: candidate columns staged in
    // shared memory (B200, config 2: DD A 167 -> 146 ms)
    p->fwd_slots = 8;
    p->fwd_staged = !p->fwd_pairs && proj_slots_valid(g.xstride, p->fwd_slots) &&
                    proj_staged_smem_bytes(G.nv, G.nx, G.ny, g.xstride, p->fwd_groups, p->fwd_rows, p->fwd_slots) <=
                        200 * 1024;
    if (p->fwd_ok)
        CTSIM_ALLOC(p->d_xs, sizeof(float) * (size_t)nxy * (p->xs_holds_pairs ? 2 * (G.nz + 1) : g.xstride));
    // the backprojection scratch (an FP32 copy of the sinogram times ampv) is allocated on
    // first use (ensure_scratch): BF16/FP16 sinograms and CTSIM_INPUT_SCALED residuals are
    // read as they are and never need it
#undef CTSIM_ALLOC
    p->bytes = bytes;
    if ((e = ctsim_plan_upload(p, p->d_views, views.data(), sizeof(View) * G.noviews)) != cudaSuccess ||
        (e = ctsim_plan_upload(p, p->d_ampv, ampv.data(), sizeof(float) * ampv.size())) != cudaSuccess ||
        (e = ctsim_plan_upload(p, p->d_map, mp.data(), mp.size())) != cudaSuccess ||
        (e = stream_ordered ? cudaMemsetAsync(p->d_err, 0, sizeof(int), stream)
                            : cudaMemset(p->d_err, 0, sizeof(int))) != cudaSuccess) {
        free_plan(p);
        return cuda_fail(e, "plan upload");
    }
    *out = p;
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_plan_destroy(ctsim_plan *plan) {
    free_plan(plan);
    return CTSIM_OK;
}

extern "C" size_t ctsim_plan_device_bytes(const ctsim_plan *plan) { return plan ? plan->bytes : 0; }

static ctsim_status check_views(const ctsim_plan *p, int vb, int vs, int vc) {
    if (vc < 1 || vs < 1 || vb < 0 || (long long)vb + (long long)(vc - 1) * vs >= p->geom.noviews)
        return fail(CTSIM_ERR_ARGUMENT, "view selection outside the plan's views");
    return CTSIM_OK;
}

static bool dtype_ok(int d) { return d == CTSIM_F32 || d == CTSIM_BF16 || d == CTSIM_F16; }

static const char *kArcOnlyDD =
    "the arc detector (detector_type 2) is defined for the distance-driven pair only (geom/cbct/cbct_proj3.c)";

static ctsim_status plan_project(ctsim_plan *p, int method, const void *d_image, int image_dtype, void *d_proj,
                                 int proj_dtype, int view_begin, int view_stride, int view_count, void *stream,
                                 bool prefix);

extern "C" ctsim_status ctsim_plan_project_ex(ctsim_plan *p, int method, const void *d_image, int image_dtype,
                                              void *d_proj, int proj_dtype, int view_begin, int view_stride,
                                              int view_count, void *stream) {
    return plan_project(p, method, d_image, image_dtype, d_proj, proj_dtype, view_begin, view_stride, view_count,
                        stream, true);
}

// The backprojection scratch d_ps ([noviews][nu][nv] FP32), allocated with the plan's own
// allocation mode at the first call that needs it: a DD/SF A^T of an unscaled FP32 sinogram
// (the sinogram times ampv goes there first).  Not during stream capture: a plan that
// will be captured makes one such call before.
static ctsim_status ensure_scratch(ctsim_plan *p, cudaStream_t st) {
    if (p->d_ps) return CTSIM_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (st && cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
        return fail(CTSIM_ERR_ARGUMENT,
                    "the plan's first unscaled FP32 backprojection allocates its scratch: make one before stream "
                    "capture (or pass BF16/FP16 or CTSIM_INPUT_SCALED data)");
    const size_t n = sizeof(float) * (size_t)p->geom.nu * p->geom.nv * p->geom.noviews;
    void *ptr = nullptr;
    cudaError_t e = ctsim_plan_alloc(p, &ptr, n);
    if (e != cudaSuccess) return fail(CTSIM_ERR_ALLOC, std::string("backprojection scratch: ") + cudaGetErrorString(e));
    // a stream-ordered allocation is usable on the plan's stream; order `st` after it
    if (p->stream_ordered && st != p->stream && (e = cudaStreamSynchronize(p->stream)) != cudaSuccess) {
        ctsim_plan_release(p, ptr);
        return cuda_fail(e, "backprojection scratch");
    }
    p->d_ps = static_cast<float *>(ptr);
    p->bytes += n;
    return CTSIM_OK;
}

// prefix = false reuses the column prefix sums of the previous call on the same image
// (the host-pointer path projects one image in view chunks).
static ctsim_status plan_project(ctsim_plan *p, int method, const void *d_image, int image_dtype, void *d_proj,
                                 int proj_dtype, int view_begin, int view_stride, int view_count, void *stream,
                                 bool prefix) {
    if (!p || !d_image || !d_proj) return fail(CTSIM_ERR_ARGUMENT, "null argument");
    if (method != CTSIM_PROJ_DD && method != CTSIM_PROJ_TF) return fail(CTSIM_ERR_ARGUMENT, "unknown forward method");
    if (p->g.det == 2 && method != CTSIM_PROJ_DD) return fail(CTSIM_ERR_UNSUPPORTED, kArcOnlyDD);
    if (!dtype_ok(image_dtype) || !dtype_ok(proj_dtype)) return fail(CTSIM_ERR_ARGUMENT, "unknown storage type");
    ctsim_status s = check_views(p, view_begin, view_stride, view_count);
    if (s != CTSIM_OK) return s;
    if (!p->fwd_ok) return fail(CTSIM_ERR_UNSUPPORTED, p->fwd_reason);
    cudaStream_t st = (cudaStream_t)stream;
    const int nxy = p->g.nx * p->g.ny;
    cudaError_t e;
    if (prefix && (e = launch_prefix(d_image, image_dtype, p->d_xs, nxy, p->g.nz, p->fwd_pairs, p->g.xstride, st)) != cudaSuccess)
        return cuda_fail(e, "prefix kernel");
    if (p->fwd_staged && !p->fwd_pairs)
        e = launch_proj_staged(method == CTSIM_PROJ_DD ? kDD : kTF, p->fwd_groups, p->fwd_rows, p->fwd_slots, p->g,
                               p->d_views, p->d_xs, p->d_ampv, p->d_map, d_proj, proj_dtype, view_begin, view_stride,
                               view_count, p->margin, p->d_err, st);
    else
        e = launch_proj(method == CTSIM_PROJ_DD ? kDD : kTF, p->fwd_groups, p->fwd_rows, p->fwd_pairs, p->g,
                        p->d_views, p->d_xs, p->d_ampv, p->d_map, d_proj, proj_dtype, view_begin, view_stride,
                        view_count, p->margin, st);
    if (e != cudaSuccess) return cuda_fail(e, "forward projection kernel");
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_plan_project(ctsim_plan *p, int method, const float *d_image, float *d_proj,
                                           int view_begin, int view_stride, int view_count, void *stream) {
    return ctsim_plan_project_ex(p, method, d_image, CTSIM_F32, d_proj, CTSIM_F32, view_begin, view_stride,
                                 view_count, stream);
}

extern "C" ctsim_status ctsim_plan_backproject_ex(ctsim_plan *p, int method, const void *d_proj, int proj_dtype,
                                                  void *d_image, int image_dtype, int view_begin, int view_stride,
                                                  int view_count, float scale, void *stream) {
    if (!p || !d_image || !d_proj) return fail(CTSIM_ERR_ARGUMENT, "null argument");
    if (!dtype_ok(image_dtype) || !dtype_ok(proj_dtype)) return fail(CTSIM_ERR_ARGUMENT, "unknown storage type");
    const bool scaled_in = (method & CTSIM_INPUT_SCALED) != 0;
    method &= ~CTSIM_INPUT_SCALED;
    if (scaled_in && ((method != CTSIM_BACK_DD && method != CTSIM_BACK_TF) || proj_dtype != CTSIM_F32))
        return fail(CTSIM_ERR_ARGUMENT, "CTSIM_INPUT_SCALED takes an FP32 sinogram for back,dd / back,tf");
    if (p->g.det == 2 && method != CTSIM_BACK_DD) return fail(CTSIM_ERR_UNSUPPORTED, kArcOnlyDD);
    ctsim_status s = check_views(p, view_begin, view_stride, view_count);
    if (s != CTSIM_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nuv = (size_t)p->g.nu * p->g.nv;
    cudaError_t e;
    switch (method) {
    case CTSIM_BACK_DD:
    case CTSIM_BACK_TF: {
        if (!p->fwd_ok) return fail(CTSIM_ERR_UNSUPPORTED, p->fwd_reason);
        // BF16/FP16 sinograms and scaled FP32 residuals are read as they are; an unscaled
        // FP32 sinogram is multiplied by ampv into the scratch first
        const void *src = d_proj;
        int kind = proj_dtype == CTSIM_BF16 ? kSrcBF16 : proj_dtype == CTSIM_F16 ? kSrcF16 : kSrcScaled;
        if (proj_dtype == CTSIM_F32 && !scaled_in) {
            if ((s = ensure_scratch(p, st)) != CTSIM_OK) return s;
            e = launch_prescale(d_proj, proj_dtype, p->d_ampv, p->d_ps, nuv, nuv * view_count, st);
            if (e != cudaSuccess) return cuda_fail(e, "prescale kernel");
            src = p->d_ps;
        }
        const bool dd = method == CTSIM_BACK_DD;
        e = launch_back(dd ? kDD : kTF, dd ? p->back_mz : p->back_mz_tf, p->g, p->d_views, src, p->d_map, d_image,
                        image_dtype, view_begin, view_stride, view_count, scale, dd ? p->back_qcap : p->back_qcap_tf,
                        p->d_err, st, false, 0, -1, kind, p->d_ampv);
        break;
    }
    case CTSIM_BACK_PD:
    case CTSIM_BACK_HPD:
    case CTSIM_BACK_VAR: {
        // the sinogram is read in its storage type (no FP32 copy)
        const int mode = method == CTSIM_BACK_PD ? kPdOff : method == CTSIM_BACK_HPD ? kPdClamp : kPdVar;
        e = launch_pd(mode, p->pd_mz, p->g, p->d_views, d_proj, p->d_map, d_image, image_dtype, view_begin,
                      view_stride, view_count, scale, st, false, proj_dtype);
        break;
    }
    default:
        return fail(CTSIM_ERR_ARGUMENT, "unknown backprojection method");
    }
    if (e != cudaSuccess) return cuda_fail(e, "backprojection kernel");
    return CTSIM_OK;
}

// Column prefix sums of an FP32 image for the forward projection of a later plan_project
// with prefix = false.
static ctsim_status plan_prefix(ctsim_plan *p, int method, const void *d_image, cudaStream_t st) {
    if (method != CTSIM_PROJ_DD && method != CTSIM_PROJ_TF) return fail(CTSIM_ERR_ARGUMENT, "unknown forward method");
    if (p->g.det == 2 && method != CTSIM_PROJ_DD) return fail(CTSIM_ERR_UNSUPPORTED, kArcOnlyDD);
    if (!p->fwd_ok) return fail(CTSIM_ERR_UNSUPPORTED, p->fwd_reason);
    const cudaError_t e = launch_prefix(d_image, CTSIM_F32, p->d_xs, p->g.nx * p->g.ny, p->g.nz, p->fwd_pairs, p->g.xstride, st);
    return e == cudaSuccess ? CTSIM_OK : cuda_fail(e, "prefix kernel");
}

// A^T (DD or SF) of views [vb, vb + vc) of FP32 d_proj into the FP32 image, scale 1; with
// accumulate the image holds the sum over the earlier views and the kernel continues it,
// so a sinogram backprojected chunk by chunk gives the one-pass result bit for bit.
static ctsim_status plan_back_views(ctsim_plan *p, int method, const float *d_proj, float *d_image, int vb, int vc,
                                    bool accumulate, cudaStream_t st, bool prescale = true, int y_begin = 0,
                                    int y_end = -1) {
    if (p->g.det == 2 && method != CTSIM_BACK_DD) return fail(CTSIM_ERR_UNSUPPORTED, kArcOnlyDD);
    ctsim_status s = check_views(p, vb, 1, vc);
    if (s != CTSIM_OK) return s;
    if (method == CTSIM_BACK_PD || method == CTSIM_BACK_HPD || method == CTSIM_BACK_VAR) {
        // FP32 sinogram read as it is; no y slabs
        const int mode = method == CTSIM_BACK_PD ? kPdOff : method == CTSIM_BACK_HPD ? kPdClamp : kPdVar;
        const cudaError_t e = launch_pd(mode, p->pd_mz, p->g, p->d_views, d_proj, p->d_map, d_image, CTSIM_F32, vb,
                                        1, vc, 1.0f, st, accumulate);
        return e == cudaSuccess ? CTSIM_OK : cuda_fail(e, "backprojection kernel");
    }
    if (!p->fwd_ok) return fail(CTSIM_ERR_UNSUPPORTED, p->fwd_reason);
    if ((s = ensure_scratch(p, st)) != CTSIM_OK) return s;
    const size_t nuv = (size_t)p->g.nu * p->g.nv;
    cudaError_t e;
    if (prescale && (e = launch_prescale(d_proj, CTSIM_F32, p->d_ampv, p->d_ps, nuv, nuv * vc, st)) != cudaSuccess)
        return cuda_fail(e, "prescale kernel");
    const bool dd = method == CTSIM_BACK_DD;
    e = launch_back(dd ? kDD : kTF, dd ? p->back_mz : p->back_mz_tf, p->g, p->d_views, p->d_ps, p->d_map, d_image,
                    CTSIM_F32, vb, 1, vc, 1.0f, dd ? p->back_qcap : p->back_qcap_tf, p->d_err, st, accumulate,
                    y_begin, y_end);
    if (e != cudaSuccess) return cuda_fail(e, "backprojection kernel");
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_plan_backproject(ctsim_plan *p, int method, const float *d_proj, float *d_image,
                                               int view_begin, int view_stride, int view_count, float scale,
                                               void *stream) {
    return ctsim_plan_backproject_ex(p, method, d_proj, CTSIM_F32, d_image, CTSIM_F32, view_begin, view_stride,
                                     view_count, scale, stream);
}

// Synchronous check of the plan's device error flag (set if a kernel met a
// footprint larger than its buffers; never expected for a valid plan).
extern "C" ctsim_status ctsim_plan_check(ctsim_plan *p) {
    if (!p) return fail(CTSIM_ERR_ARGUMENT, "null plan");
    int h = 0;
    // stream-ordered plans: read the flag on the plan's own stream (a legacy-stream copy
    // would wait for every other request's work on the device)
    cudaError_t e = p->stream_ordered ? cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, p->stream)
                                      : cudaMemcpy(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && p->stream_ordered) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return cuda_fail(e, "error flag read");
    if (h) return fail(CTSIM_ERR_UNSUPPORTED, "a footprint exceeded the kernel's row buffer");
    return CTSIM_OK;
}

// ---------------------------------------------------------------------------
// Drop-in host-pointer entry points.
// ---------------------------------------------------------------------------
namespace {

// ---------------------------------------------------------------------------
// Host-pointer entry points.  Each call is synchronous, as the reference MEX back ends
// are.  Unlike them, the last geometry's plan, device buffers and streams stay on the
// device between calls (a reconstruction calls the gateway again and again with one
// geometry), until the geometry changes or ctsim_host_cache_release; and the data moves
// in view chunks that overlap the kernels (forward results out, backprojection inputs in).
// ---------------------------------------------------------------------------
namespace {
// Parts of a host-side job run on a small pool of threads plus the caller (the
// pageable-memory staging below: one thread's memcpy moves about 15 GB/s, eight about 50,
// while pageable cudaMemcpy moves 11 GB/s host to device on B200 hosts).  The pool is
// created on first use and never destroyed; its threads stay parked on a condition
// variable, so process exit does not wait for them.
class HostPool {
  public:
    static HostPool &get() {
        static HostPool *pool = new HostPool();
        return *pool;
    }
    int width() const { return workers_ + 1; }
    // fn(0) .. fn(n - 1), on the pool and the calling thread; returns when all are done.
    void run(int n, const std::function<void(int)> &fn) {
        std::lock_guard<std::mutex> one_job(job_m_);
        if (n <= 1 || workers_ == 0) {
            for (int i = 0; i < n; i++) fn(i);
            return;
        }
        auto job = std::make_shared<Job>();
        job->fn = &fn;
        job->n = n;
        job->left.store(n);
        {
            std::lock_guard<std::mutex> l(m_);
            job_ = job;
            gen_++;
        }
        cv_.notify_all();
        work(*job);
        std::unique_lock<std::mutex> l(job->m);
        job->cv.wait(l, [&] { return job->left.load() == 0; });
    }
    // memcpy in parts of at least 4 MB, one per pool thread at most.
    void copy(void *dst, const void *src, size_t n) {
        const int parts = (int)std::min<size_t>((size_t)width(), std::max<size_t>(1, n >> 22));
        const size_t per = ((n + parts - 1) / parts + 63) & ~(size_t)63;
        run(parts, [&](int i) {
            const size_t o = (size_t)i * per;
            if (o < n) std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, std::min(per, n - o));
        });
    }

  private:
    struct Job {
        const std::function<void(int)> *fn = nullptr;
        int n = 0;
        std::atomic<int> next{0}, left{0};
        std::mutex m;
        std::condition_variable cv;
    };
    HostPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        workers_ = (int)std::min(7u, hw > 2 ? hw / 2 - 1 : 0u);
        for (int i = 0; i < workers_; i++) std::thread([this] { loop(); }).detach();
    }
    // A worker that wakes after its job ended finds the job's parts taken and leaves it.
    static void work(Job &j) {
        for (int i; (i = j.next.fetch_add(1)) < j.n;) {
            (*j.fn)(i);
            if (j.left.fetch_sub(1) == 1) {
                std::lock_guard<std::mutex> l(j.m);
                j.cv.notify_all();
            }
        }
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> l(m_);
                cv_.wait(l, [&] { return gen_ != seen; });
                seen = gen_;
                job = job_;
            }
            work(*job);
        }
    }
    int workers_ = 0;
    std::mutex job_m_, m_;
    std::condition_variable cv_;
    std::shared_ptr<Job> job_;
    unsigned long long gen_ = 0;
};

// First view of chunk c (0 .. nch) when n views are split into nch chunks for the host
// path.  With enough views one chunk, the first (A^T: its copy in cannot overlap compute)
// or the last (A: its copy out cannot), gets a quarter of the others' views, so the
// copies outside the overlap are short.  Every chunk keeps at least two views.
int chunk_first_view(int n, int nch, int c, bool small_last) {
    if (n < 8 * nch || nch < 2) return (int)((long long)n * c / nch);
    const long long total = 4LL * (nch - 1) + 1;  // weight 1 for the short chunk, 4 for the others
    const long long w = small_last ? (c == nch ? total : 4LL * c) : (c == 0 ? 0 : 1 + 4LL * (c - 1));
    return (int)((long long)n * w / total);
}

// True for page-locked (registered or cudaHostAlloc'd) host memory and device memory;
// false for ordinary pageable memory.
bool dma_ready(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

struct HostCache {
    std::mutex m;
    int device = -1;
    ctsim_geom G{};
    std::vector<double> betas;
    std::vector<float> couch;
    std::vector<uint8_t> map;  // empty: no map
    ctsim_plan *plan = nullptr;
    void *dimg = nullptr, *dsino = nullptr;
    cudaStream_t st = nullptr, st2 = nullptr, copy = nullptr;
    static constexpr int kChunks = 8;  // view chunks of a call
    static constexpr int kSlabs = 4;   // y slabs of the last backprojection chunk
    cudaEvent_t done[kChunks + kSlabs] = {};
    cudaEvent_t ready = nullptr;
    // pinned staging for pageable caller buffers: kStage buffers of kStageBytes, each with
    // the event of the last copy that used it (allocated on the first pageable call)
    static constexpr int kStage = 4;
    static constexpr size_t kStageBytes = (size_t)32 << 20;
    void *stage[kStage] = {};
    cudaEvent_t stage_ev[kStage] = {};

    cudaError_t ensure_stage() {
        if (stage[0]) return cudaSuccess;
        cudaError_t e = cudaSuccess;
        for (int b = 0; b < kStage && e == cudaSuccess; b++)
            if ((e = cudaHostAlloc(&stage[b], kStageBytes, cudaHostAllocDefault)) == cudaSuccess)
                e = cudaEventCreateWithFlags(&stage_ev[b], cudaEventDisableTiming);
        if (e != cudaSuccess) release_stage();
        return e;
    }
    void release_stage() {
        for (int b = 0; b < kStage; b++) {
            if (stage_ev[b]) cudaEventSynchronize(stage_ev[b]);
            if (stage[b]) cudaFreeHost(stage[b]);
            if (stage_ev[b]) cudaEventDestroy(stage_ev[b]);
            stage[b] = nullptr;
            stage_ev[b] = nullptr;
        }
    }
    // Host to device from pageable src through the staging buffers, in order on stream s:
    // the pool fills one buffer while the copy engine drains the previous one.  Returns
    // once the last piece is queued (src may then be reused).
    cudaError_t staged_h2d(void *dst, const void *src, size_t n, cudaStream_t s) {
        cudaError_t e;
        for (size_t off = 0, i = 0; off < n; off += kStageBytes, i++) {
            const int b = (int)(i % kStage);
            const size_t len = std::min(kStageBytes, n - off);
            if ((e = cudaEventSynchronize(stage_ev[b])) != cudaSuccess) return e;  // its last copy is done
            HostPool::get().copy(stage[b], static_cast<const char *>(src) + off, len);
            if ((e = cudaMemcpyAsync(static_cast<char *>(dst) + off, stage[b], len, cudaMemcpyHostToDevice, s)) !=
                    cudaSuccess ||
                (e = cudaEventRecord(stage_ev[b], s)) != cudaSuccess)
                return e;
        }
        return cudaSuccess;
    }
    // Device to pageable host after the work queued on stream s: up to kStage pieces in
    // flight, each copied out by the pool as it lands.  Returns when dst holds the data.
    cudaError_t staged_d2h(void *dst, const void *src, size_t n, cudaStream_t s) {
        const size_t np = (n + kStageBytes - 1) / kStageBytes;
        cudaError_t e;
        auto issue = [&](size_t i) {
            const int b = (int)(i % kStage);
            const size_t off = i * kStageBytes, len = std::min(kStageBytes, n - off);
            cudaError_t r;
            if ((r = cudaStreamWaitEvent(s, stage_ev[b], 0)) != cudaSuccess ||
                (r = cudaMemcpyAsync(stage[b], static_cast<const char *>(src) + off, len, cudaMemcpyDeviceToHost, s)) !=
                    cudaSuccess)
                return r;
            return cudaEventRecord(stage_ev[b], s);
        };
        for (size_t i = 0; i < std::min<size_t>(kStage, np); i++)
            if ((e = issue(i)) != cudaSuccess) return e;
        for (size_t i = 0; i < np; i++) {
            const int b = (int)(i % kStage);
            const size_t off = i * kStageBytes, len = std::min(kStageBytes, n - off);
            if ((e = cudaEventSynchronize(stage_ev[b])) != cudaSuccess) return e;
            HostPool::get().copy(static_cast<char *>(dst) + off, stage[b], len);
            if (i + kStage < np && (e = issue(i + kStage)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    void release() {
        int cur = -1;
        if (device >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != device) cudaSetDevice(device);
        if (plan) ctsim_plan_destroy(plan);
        plan = nullptr;
        cudaFree(dimg);
        cudaFree(dsino);
        dimg = dsino = nullptr;
        for (auto &e : done) {
            if (e) cudaEventDestroy(e);
            e = nullptr;
        }
        if (ready) cudaEventDestroy(ready);
        ready = nullptr;
        release_stage();
        for (cudaStream_t s : {st, st2, copy})
            if (s) cudaStreamDestroy(s);
        st = st2 = copy = nullptr;
        if (cur >= 0 && cur != device) cudaSetDevice(cur);
        device = -1;
    }
    bool matches(int dev, const ctsim_geom &g, const double *b, const float *c, const bool *mp) const {
        if (!plan || dev != device || std::memcmp(&g, &G, sizeof(G)) != 0) return false;
        if (std::memcmp(b, betas.data(), sizeof(double) * g.noviews) || std::memcmp(c, couch.data(), sizeof(float) * g.noviews))
            return false;
        if ((mp == nullptr) != map.empty()) return false;
        if (mp)
            for (size_t i = 0; i < map.size(); i++)
                if ((mp[i] ? 1 : 0) != map[i]) return false;
        return true;
    }
    cudaError_t set_up(int dev, const ctsim_geom &g, const double *b, const float *c, const bool *mp, bool *ok) {
        release();
        *ok = false;
        if (ctsim_plan_create(&g, b, c, mp, &plan) != CTSIM_OK) return cudaSuccess;  // message already set
        const size_t nimg = (size_t)g.nx * g.ny * g.nz, nsino = (size_t)g.nu * g.nv * g.noviews;
        cudaError_t e;
        if ((e = cudaMalloc(&dimg, nimg * sizeof(float))) != cudaSuccess ||
            (e = cudaMalloc(&dsino, nsino * sizeof(float))) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming)) != cudaSuccess)
            return e;
        for (auto &ev : done)
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
        device = dev;
        G = g;
        betas.assign(b, b + g.noviews);
        couch.assign(c, c + g.noviews);
        map.clear();
        if (mp) {
            map.resize((size_t)g.nx * g.ny);
            for (size_t i = 0; i < map.size(); i++) map[i] = mp[i] ? 1 : 0;
        }
        *ok = true;
        return cudaSuccess;
    }
};
// One cache per device, so that threads driving different GPUs neither wait for nor
// evict each other.
std::mutex g_host_map_m;
std::map<int, std::unique_ptr<HostCache>> g_host_by_dev;
std::atomic<bool> g_host_enabled{true};

HostCache &host_cache(int dev) {
    std::lock_guard<std::mutex> lock(g_host_map_m);
    std::unique_ptr<HostCache> &c = g_host_by_dev[dev];
    if (!c) c.reset(new HostCache);
    return *c;
}

void release_host_caches() {
    std::lock_guard<std::mutex> lock(g_host_map_m);
    for (auto &kv : g_host_by_dev) {
        std::lock_guard<std::mutex> l(kv.second->m);
        kv.second->release();
    }
}
}  // namespace

bool run_host(int method, const ctsim_geom &G, const double *betas, const float *couchz, const bool *map,
              const float *in, float *out) {
    if (!betas || !couchz || !in || !out) {
        fail(CTSIM_ERR_ARGUMENT, "null argument");
        return false;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        fail(CTSIM_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
        return false;
    }
    HostCache &h = host_cache(dev);
    std::lock_guard<std::mutex> lock(h.m);
    if (!h.matches(dev, G, betas, couchz, map)) {
        bool made = false;
        if ((e = h.set_up(dev, G, betas, couchz, map, &made)) != cudaSuccess) {
            h.release();
            fail(CTSIM_ERR_ALLOC, std::string("device set-up: ") + cudaGetErrorString(e));
            return false;
        }
        if (!made) {
            h.release();
            return false;
        }
    }
    ctsim_plan *p = h.plan;
    const bool fwd = method == CTSIM_PROJ_DD || method == CTSIM_PROJ_TF;
    const size_t nimg = (size_t)G.nx * G.ny * G.nz, nuv = (size_t)G.nu * G.nv, nsino = nuv * G.noviews;
    // pageable caller buffers go through the pinned staging buffers (if they can be had;
    // otherwise the driver stages them)
    bool stage_in = !dma_ready(in), stage_out = !dma_ready(out);
    if ((stage_in || stage_out) && h.ensure_stage() != cudaSuccess) {
        cudaGetLastError();
        stage_in = stage_out = false;
    }
    auto h2d = [&](void *dst, const void *src, size_t n, cudaStream_t st) {
        return stage_in ? h.staged_h2d(dst, src, n, st) : cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st);
    };
    bool ok = false;
    do {
        if (fwd) {
            // the image and its column prefix sums, then the views in chunks on two compute
            // streams (one chunk's tail overlaps the next one's start); each chunk's sinogram is
            // copied back on the copy stream while later chunks compute (the views are
            // independent).  All chunks are queued before the first copy: a copy to pageable
            // memory returns only when it has finished.
            if ((e = h2d(h.dimg, in, nimg * sizeof(float), h.st)) != cudaSuccess) {
                cuda_fail(e, "host to device copy");
                break;
            }
            ctsim_status s = plan_prefix(p, method, h.dimg, h.st);
            if (s == CTSIM_OK && ((e = cudaEventRecord(h.ready, h.st)) != cudaSuccess ||
                                  (e = cudaStreamWaitEvent(h.st2, h.ready, 0)) != cudaSuccess))
                s = cuda_fail(e, "event");
            const int nch = std::min(HostCache::kChunks, G.noviews);
            auto first_view = [&](int c) { return chunk_first_view(G.noviews, nch, c, true); };
            for (int c = 0; c < nch && s == CTSIM_OK; c++) {
                const int vb = first_view(c), ve = first_view(c + 1);
                cudaStream_t sc = (c & 1) ? h.st2 : h.st;
                float *dproj = static_cast<float *>(h.dsino) + (size_t)vb * nuv;
                s = plan_project(p, method, h.dimg, CTSIM_F32, dproj, CTSIM_F32, vb, 1, ve - vb, sc, false);
                if (s == CTSIM_OK && (e = cudaEventRecord(h.done[c], sc)) != cudaSuccess) s = cuda_fail(e, "event");
            }
            for (int c = 0; c < nch && s == CTSIM_OK; c++) {
                const int vb = first_view(c), ve = first_view(c + 1);
                float *hdst = out + (size_t)vb * nuv;
                const float *dsrc = static_cast<float *>(h.dsino) + (size_t)vb * nuv;
                const size_t bytes = (size_t)(ve - vb) * nuv * sizeof(float);
                if ((e = cudaStreamWaitEvent(h.copy, h.done[c], 0)) != cudaSuccess ||
                    (e = stage_out ? h.staged_d2h(hdst, dsrc, bytes, h.copy)
                                   : cudaMemcpyAsync(hdst, dsrc, bytes, cudaMemcpyDeviceToHost, h.copy)) != cudaSuccess)
                    s = cuda_fail(e, "device to host copy");
            }
            const cudaError_t e1 = cudaStreamSynchronize(h.st), e2 = cudaStreamSynchronize(h.st2),
                              e3 = cudaStreamSynchronize(h.copy);
            if (s != CTSIM_OK) break;
            if ((e = e1) != cudaSuccess || (e = e2) != cudaSuccess || (e = e3) != cudaSuccess) {
                cuda_fail(e, "kernel execution");
                break;
            }
        } else if (method == CTSIM_BACK_DD || method == CTSIM_BACK_TF || method == CTSIM_BACK_PD ||
                   method == CTSIM_BACK_HPD || method == CTSIM_BACK_VAR) {
            // the sinogram in view chunks on the copy stream; each chunk is backprojected,
            // continuing the image's view sums, while the next one is copied in.  For DD/SF
            // the last chunk runs in y slabs, and each finished slab goes back to the host
            // while the next one computes (voxels are independent).
            // (a staged, pageable image goes back in one piece after the last chunk)
            const bool slabs = (method == CTSIM_BACK_DD || method == CTSIM_BACK_TF) && !stage_out;
            const int nch = std::min(HostCache::kChunks, G.noviews);
            auto first_view = [&](int c) { return chunk_first_view(G.noviews, nch, c, false); };
            auto first_row = [&](int k) { return (int)((long long)G.ny * k / HostCache::kSlabs); };
            ctsim_status s = CTSIM_OK;
            for (int c = 0; c < nch && s == CTSIM_OK; c++) {
                const int vb = first_view(c), ve = first_view(c + 1);
                float *dproj = static_cast<float *>(h.dsino) + (size_t)vb * nuv;
                if ((e = h2d(dproj, in + (size_t)vb * nuv, (size_t)(ve - vb) * nuv * sizeof(float), h.copy)) !=
                        cudaSuccess ||
                    (e = cudaEventRecord(h.done[c], h.copy)) != cudaSuccess ||
                    (e = cudaStreamWaitEvent(h.st, h.done[c], 0)) != cudaSuccess) {
                    s = cuda_fail(e, "host to device copy");
                    break;
                }
                if (c + 1 < nch || !slabs) {
                    s = plan_back_views(p, method, dproj, static_cast<float *>(h.dimg), vb, ve - vb, c > 0, h.st);
                    continue;
                }
                for (int k = 0; k < HostCache::kSlabs && s == CTSIM_OK; k++) {
                    s = plan_back_views(p, method, dproj, static_cast<float *>(h.dimg), vb, ve - vb, c > 0, h.st,
                                        k == 0, first_row(k), first_row(k + 1));
                    if (s == CTSIM_OK && (e = cudaEventRecord(h.done[HostCache::kChunks + k], h.st)) != cudaSuccess)
                        s = cuda_fail(e, "event");
                }
            }
            const size_t plane = (size_t)G.nx * G.ny;
            if (!slabs && s == CTSIM_OK &&
                (e = stage_out ? h.staged_d2h(out, h.dimg, nimg * sizeof(float), h.st)
                               : cudaMemcpyAsync(out, h.dimg, nimg * sizeof(float), cudaMemcpyDeviceToHost, h.st)) !=
                    cudaSuccess)
                s = cuda_fail(e, "device to host copy");
            for (int k = 0; slabs && k < HostCache::kSlabs && s == CTSIM_OK; k++) {
                const int y0 = first_row(k), y1 = first_row(k + 1);
                if (y1 == y0) continue;
                if ((e = cudaStreamWaitEvent(h.copy, h.done[HostCache::kChunks + k], 0)) != cudaSuccess ||
                    (e = cudaMemcpy2DAsync(out + (size_t)y0 * G.nx, plane * sizeof(float),
                                           static_cast<float *>(h.dimg) + (size_t)y0 * G.nx, plane * sizeof(float),
                                           (size_t)(y1 - y0) * G.nx * sizeof(float), G.nz, cudaMemcpyDeviceToHost,
                                           h.copy)) != cudaSuccess)
                    s = cuda_fail(e, "device to host copy");
            }
            const cudaError_t e1 = cudaStreamSynchronize(h.st), e2 = cudaStreamSynchronize(h.copy);
            if (s != CTSIM_OK) break;
            if ((e = e1) != cudaSuccess || (e = e2) != cudaSuccess) {
                cuda_fail(e, "kernel execution");
                break;
            }
        } else {
            if ((e = cudaMemcpyAsync(h.dsino, in, nsino * sizeof(float), cudaMemcpyHostToDevice, h.st)) != cudaSuccess) {
                cuda_fail(e, "host to device copy");
                break;
            }
            if (ctsim_plan_backproject(p, method, (const float *)h.dsino, (float *)h.dimg, 0, 1, G.noviews, 1.0f,
                                       h.st) != CTSIM_OK)
                break;
            if ((e = cudaMemcpyAsync(out, h.dimg, nimg * sizeof(float), cudaMemcpyDeviceToHost, h.st)) != cudaSuccess) {
                cuda_fail(e, "device to host copy");
                break;
            }
            if ((e = cudaStreamSynchronize(h.st)) != cudaSuccess) {
                cuda_fail(e, "kernel execution");
                break;
            }
        }
        if (ctsim_plan_check(p) != CTSIM_OK) break;
        ok = true;
    } while (0);
    if (!ok || !g_host_enabled.load()) h.release();  // after an error, nothing of the failed call is kept
    return ok;
}

ctsim_geom make_geom(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz, int nu,
                     int nv, float du, float dv, float ou, float ov, float sad, float add, float sdd, int noviews,
                     int detector_type) {
    ctsim_geom G;
    G.nx = nx; G.ny = ny; G.nz = nz; G.dx = dx; G.dy = dy; G.dz = dz;
    G.offset_x = ox; G.offset_y = oy; G.offset_z = oz;
    G.nu = nu; G.nv = nv; G.du = du; G.dv = dv; G.offset_u = ou; G.offset_v = ov;
    G.sad = sad; G.add = add; G.sdd = sdd; G.noviews = noviews; G.detector_type = detector_type;
    return G;
}

}  // namespace

extern "C" ctsim_status ctsim_host_cache_release(void) {
    release_host_caches();
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_host_cache_enable(int enabled) {
    g_host_enabled.store(enabled != 0);
    if (!enabled) release_host_caches();
    return CTSIM_OK;
}

#define CTSIM_GEOM_PARAMS                                                                                        \
    int nx, int ny, int nz, float dx, float dy, float dz, float offset_x, float offset_y, float offset_z, int nu, \
        int nv, float du, float dv, float offset_u, float offset_v, float sad, float add, float sdd, int noviews, \
        const double *betas, const float *couchz, int detector_type
#define CTSIM_GEOM_VALUES \
    make_geom(nx, ny, nz, dx, dy, dz, offset_x, offset_y, offset_z, nu, nv, du, dv, offset_u, offset_v, sad, add, sdd, noviews, detector_type)

extern "C" bool ctsim_proj_dd(CTSIM_GEOM_PARAMS, const float *image, float *proj, const bool *map) {
    return run_host(CTSIM_PROJ_DD, CTSIM_GEOM_VALUES, betas, couchz, map, image, proj);
}
extern "C" bool ctsim_proj_tf(CTSIM_GEOM_PARAMS, const float *image, float *proj, const bool *map) {
    return run_host(CTSIM_PROJ_TF, CTSIM_GEOM_VALUES, betas, couchz, map, image, proj);
}
extern "C" bool ctsim_back_dd(CTSIM_GEOM_PARAMS, float *image, const float *proj, const bool *map) {
    return run_host(CTSIM_BACK_DD, CTSIM_GEOM_VALUES, betas, couchz, map, proj, image);
}
extern "C" bool ctsim_back_tf(CTSIM_GEOM_PARAMS, float *image, const float *proj, const bool *map) {
    return run_host(CTSIM_BACK_TF, CTSIM_GEOM_VALUES, betas, couchz, map, proj, image);
}
extern "C" bool ctsim_back_pd(CTSIM_GEOM_PARAMS, float *image, const float *proj, const bool *map, bool offBoundary) {
    return run_host(offBoundary ? CTSIM_BACK_PD : CTSIM_BACK_HPD, CTSIM_GEOM_VALUES, betas, couchz, map, proj, image);
}

extern "C" bool ctsim_cbct_geom(const char *type, CTSIM_GEOM_PARAMS, const float *data, float *out, const bool *map) {
    if (!type) {
        fail(CTSIM_ERR_ARGUMENT, "The 1st argument is invalid!");
        return false;
    }
    // string dispatch of geom/cbct/cbct_geom_mex.c:267-306 ("proj,rd" and "back,var" are not provided)
    int method = -1;
    if (!std::strcmp(type, "proj,dd")) method = CTSIM_PROJ_DD;
    else if (!std::strcmp(type, "proj,tf")) method = CTSIM_PROJ_TF;
    else if (!std::strcmp(type, "back,dd")) method = CTSIM_BACK_DD;
    else if (!std::strcmp(type, "back,tf")) method = CTSIM_BACK_TF;
    else if (!std::strcmp(type, "back,pd")) method = CTSIM_BACK_PD;
    else if (!std::strcmp(type, "back,hpd")) method = CTSIM_BACK_HPD;
    else if (!std::strcmp(type, "back,var")) method = CTSIM_BACK_VAR;
    if (method < 0) {
        fail(CTSIM_ERR_ARGUMENT, "Error: unknown geom type.");
        return false;
    }
    return run_host(method, CTSIM_GEOM_VALUES, betas, couchz, map, data, out);
}

// ---------------------------------------------------------------------------
// Tuning: the forward projector's candidate groups, the A^T and FDK z-pass depths.
// ---------------------------------------------------------------------------
extern "C" ctsim_status ctsim_plan_get_tuning(const ctsim_plan *p, ctsim_tuning *t) {
    if (!p || !t) return fail(CTSIM_ERR_ARGUMENT, "null argument");
    t->proj_groups = p->fwd_groups;
    t->proj_rows = p->fwd_rows;
    t->proj_layout = p->fwd_pairs ? 2 : p->fwd_staged ? 3 : 1;
    t->proj_slots = p->fwd_slots;
    t->back_mz = p->back_mz;
    t->back_mz_tf = p->back_mz_tf;
    t->pd_mz = p->pd_mz;
    return CTSIM_OK;
}

static bool mz_valid(int mz) { return mz == 1 || mz == 2 || mz == 4 || mz == 8; }

extern "C" ctsim_status ctsim_plan_set_tuning(ctsim_plan *p, const ctsim_tuning *t) {
    if (!p || !t) return fail(CTSIM_ERR_ARGUMENT, "null argument");
    if (t->proj_groups || t->proj_rows) {
        const int G = t->proj_groups ? t->proj_groups : p->fwd_groups;
        const int R = t->proj_rows ? t->proj_rows : p->fwd_rows;
        if (!proj_shape_valid(p->geom.nv, G, R) || proj_smem_bytes(p->geom.nv, p->geom.nx, p->geom.ny, G, R) > 200 * 1024)
            return fail(CTSIM_ERR_ARGUMENT,
                        "proj_groups must be 1, 2, 4 or 8 and proj_rows a multiple of 32 up to the rows' need, "
                        "with groups * rows <= 256");
    }
    if ((t->back_mz && (!mz_valid(t->back_mz) || !back_mz_fits(p, t->back_mz))) ||
        (t->back_mz_tf && (!mz_valid(t->back_mz_tf) || !back_mz_fits(p, t->back_mz_tf))))
        return fail(CTSIM_ERR_ARGUMENT, "back_mz must be 1, 2, 4 or 8 and fit the row buffer");
    if (t->pd_mz && !mz_valid(t->pd_mz)) return fail(CTSIM_ERR_ARGUMENT, "pd_mz must be 1, 2, 4 or 8");
    if (t->proj_layout && t->proj_layout != 1 && t->proj_layout != 3 && !(t->proj_layout == 2 && p->xs_holds_pairs))
        return fail(CTSIM_ERR_ARGUMENT,
                    "proj_layout must be 1 (sums), 2 (pairs, on a plan whose volume fits them) or 3 (staged sums)");
    {
        const bool staged = t->proj_layout ? t->proj_layout == 3 : (p->fwd_staged && !p->fwd_pairs);
        const int G = t->proj_groups ? t->proj_groups : p->fwd_groups;
        const int R = t->proj_rows ? t->proj_rows : p->fwd_rows;
        const int S = t->proj_slots ? t->proj_slots : p->fwd_slots;
        if (t->proj_slots && !proj_slots_valid(p->g.xstride, t->proj_slots))
            return fail(CTSIM_ERR_ARGUMENT, "proj_slots must be 1 .. 64 with slots * column bytes < 1 MiB");
        if (staged && proj_staged_smem_bytes(p->geom.nv, p->geom.nx, p->geom.ny, p->g.xstride, G, R, S) > 200 * 1024)
            return fail(CTSIM_ERR_ARGUMENT, "the staged forward projector's shared memory exceeds 200 KiB: fewer slots");
    }
    if (t->proj_groups) p->fwd_groups = t->proj_groups;
    if (t->proj_rows) p->fwd_rows = t->proj_rows;
    if (t->proj_slots) p->fwd_slots = t->proj_slots;
    if (t->proj_layout) {
        p->fwd_pairs = t->proj_layout == 2;
        p->fwd_staged = t->proj_layout == 3;
    }
    if (t->back_mz) {
        p->back_mz = t->back_mz;
        p->back_qcap = back_qcap_for(p, t->back_mz);
    }
    if (t->back_mz_tf) {
        p->back_mz_tf = t->back_mz_tf;
        p->back_qcap_tf = back_qcap_for(p, t->back_mz_tf);
    }
    if (t->pd_mz) p->pd_mz = t->pd_mz;
    return CTSIM_OK;
}

namespace {
// Choices measured in this process, by shape class: method, the volume and detector
// sizes and the detector type.
std::mutex g_tune_mutex;
std::map<std::vector<int>, ctsim_tuning> g_tuned;
}  // namespace

extern "C" ctsim_status ctsim_autotune_clear(void) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tuned.clear();
    return CTSIM_OK;
}

// The launch shapes the autotuner tries for a method (only the method's own fields set).
static std::vector<ctsim_tuning> tuning_candidates(const ctsim_plan *p, int method) {
    std::vector<ctsim_tuning> out;
    const ctsim_geom &G = p->geom;
    if (method == CTSIM_PROJ_DD || method == CTSIM_PROJ_TF) {
        const int rmax = proj_default_rows(G.nv);
        std::vector<int> rows = {rmax};
        if (rmax > 64) rows.push_back(64);
        if (rmax > 32) rows.push_back(32);
        for (int R : rows) {
            for (int Gr : {1, 2, 4, 8})
                if (proj_shape_valid(G.nv, Gr, R) && proj_smem_bytes(G.nv, G.nx, G.ny, Gr, R) <= 200 * 1024) {
                    for (int lay = p->xs_holds_pairs ? 2 : 1; lay >= 1; lay--) {
                        ctsim_tuning t = {Gr, 0, 0, 0, R, lay, 0};
                        out.push_back(t);
                    }
                    for (int S : {8, 16, 32})
                        if (proj_slots_valid(p->g.xstride, S) &&
                            proj_staged_smem_bytes(G.nv, G.nx, G.ny, p->g.xstride, Gr, R, S) <= 200 * 1024) {
                            ctsim_tuning t = {Gr, 0, 0, 0, R, 3, S};
                            out.push_back(t);
                        }
                }
        }
        return out;
    }
    for (int mz : {1, 2, 4, 8}) {
        ctsim_tuning t = {0, 0, 0, 0, 0, 0, 0};
        if (method == CTSIM_BACK_DD) { if (!back_mz_fits(p, mz)) continue; t.back_mz = mz; }
        else if (method == CTSIM_BACK_TF) { if (!back_mz_fits(p, mz)) continue; t.back_mz_tf = mz; }
        else t.pd_mz = mz;
        out.push_back(t);
    }
    return out;
}

extern "C" ctsim_status ctsim_plan_autotune(ctsim_plan *p, int method, int sample_views, void *stream,
                                            ctsim_tuning *chosen) {
    if (!p) return fail(CTSIM_ERR_ARGUMENT, "null plan");
    if (method < CTSIM_PROJ_DD || method > CTSIM_BACK_VAR) return fail(CTSIM_ERR_ARGUMENT, "unknown method");
    const bool fwd = method == CTSIM_PROJ_DD || method == CTSIM_PROJ_TF;
    const bool vox = method >= CTSIM_BACK_PD;
    if ((fwd || !vox) && !p->fwd_ok) return fail(CTSIM_ERR_UNSUPPORTED, p->fwd_reason);
    if (p->g.det == 2 && method != CTSIM_PROJ_DD && method != CTSIM_BACK_DD) return fail(CTSIM_ERR_UNSUPPORTED, kArcOnlyDD);
    const ctsim_geom &G = p->geom;
    const std::vector<int> key = {method, G.nx, G.ny, G.nz, G.nu, G.nv, G.detector_type};
    bool have = false;
    ctsim_tuning best = {0, 0, 0, 0, 0, 0, 0};
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            best = it->second;
            have = true;
        }
    }
    if (!have) {
        const std::vector<ctsim_tuning> cand = tuning_candidates(p, method);
        // the launch shape that wins depends on the grid, so the sample should be the size
        // of the real launches (an OS-PWLS subset, or all views); default: up to 64 views
        if (sample_views < 1) sample_views = 64;
        const int count = std::min(sample_views, G.noviews);
        const int stride = std::max(1, G.noviews / count);
        cudaStream_t st = (cudaStream_t)stream;
        const size_t nimg = (size_t)G.nx * G.ny * G.nz, nsino = (size_t)count * G.nu * G.nv;
        void *img = nullptr, *sino = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaError_t e;
        // the plan's own allocation mode; the buffers are freed before returning
        if ((e = ctsim_plan_alloc(p, &img, nimg * 4)) != cudaSuccess ||
            (e = ctsim_plan_alloc(p, &sino, nsino * 4)) != cudaSuccess) {
            ctsim_plan_release(p, img);
            return fail(CTSIM_ERR_ALLOC, std::string("autotune buffers: ") + cudaGetErrorString(e));
        }
        ctsim_tuning saved;
        ctsim_plan_get_tuning(p, &saved);
        float best_ms = 0.f;
        ctsim_status s = CTSIM_OK;
        if ((e = cudaMemsetAsync(img, 0, nimg * 4, st)) != cudaSuccess ||
            (e = cudaMemsetAsync(sino, 0, nsino * 4, st)) != cudaSuccess || (e = cudaEventCreate(&e0)) != cudaSuccess ||
            (e = cudaEventCreate(&e1)) != cudaSuccess) {
            s = cuda_fail(e, "autotune set-up");
        }
        for (size_t i = 0; s == CTSIM_OK && i < cand.size(); i++) {
            if ((s = ctsim_plan_set_tuning(p, &cand[i])) != CTSIM_OK) break;
            float ms = 0.f;
            for (int rep = 0; rep < 3 && s == CTSIM_OK; rep++) {  // one warm-up, then the faster of two
                cudaEventRecord(e0, st);
                s = fwd ? ctsim_plan_project(p, method, (const float *)img, (float *)sino, 0, stride, count, stream)
                        : ctsim_plan_backproject(p, method, (const float *)sino, (float *)img, 0, stride, count, 1.0f,
                                                 stream);
                cudaEventRecord(e1, st);
                if (s != CTSIM_OK) break;
                if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
                    s = cuda_fail(e, "autotune timing");
                    break;
                }
                float t_ms = 0.f;
                cudaEventElapsedTime(&t_ms, e0, e1);
                if (rep == 1 || (rep == 2 && t_ms < ms)) ms = t_ms;
            }
            if (s == CTSIM_OK && (!have || ms < best_ms)) {
                best = cand[i];
                best_ms = ms;
                have = true;
            }
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        ctsim_plan_release(p, img);
        ctsim_plan_release(p, sino);
        ctsim_plan_set_tuning(p, &saved);
        if (s != CTSIM_OK) return s;
        if (!have) return fail(CTSIM_ERR_UNSUPPORTED, "no valid launch shape");
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[key] = best;
    }
    ctsim_status s = ctsim_plan_set_tuning(p, &best);
    if (s == CTSIM_OK && chosen) ctsim_plan_get_tuning(p, chosen);
    return s;
}

// ---------------------------------------------------------------------------
// Batched launches over many plans (ctsim_batch_item).
// ---------------------------------------------------------------------------
static ctsim_status batch_check(int method, const ctsim_batch_item *items, int n, bool fwd) {
    if (!items || n < 0) return fail(CTSIM_ERR_ARGUMENT, "null batch");
    if (fwd ? (method != CTSIM_PROJ_DD && method != CTSIM_PROJ_TF) : (method != CTSIM_BACK_DD && method != CTSIM_BACK_TF))
        return fail(CTSIM_ERR_ARGUMENT, "batched launches cover the DD and SF A / A^T");
    int dev = -1;
    for (int i = 0; i < n; i++) {
        const ctsim_batch_item &it = items[i];
        if (!it.plan || !it.in || !it.out) return fail(CTSIM_ERR_ARGUMENT, "null plan or buffer in the batch");
        if (!dtype_ok(it.in_dtype) || !dtype_ok(it.out_dtype)) return fail(CTSIM_ERR_ARGUMENT, "unknown storage type");
        if (!it.plan->fwd_ok) return fail(CTSIM_ERR_UNSUPPORTED, it.plan->fwd_reason);
        if (it.plan->g.det == 2 && method != (fwd ? CTSIM_PROJ_DD : CTSIM_BACK_DD))
            return fail(CTSIM_ERR_UNSUPPORTED, kArcOnlyDD);
        if (dev >= 0 && it.plan->device != dev) return fail(CTSIM_ERR_ARGUMENT, "batch plans must share one device");
        for (int j = 0; j < i; j++)  // each plan's scratch serves one item
            if (items[j].plan == it.plan) return fail(CTSIM_ERR_ARGUMENT, "a plan may appear only once per batch");
        dev = it.plan->device;
        ctsim_status s = check_views(it.plan, it.view_begin, it.view_stride, it.view_count);
        if (s != CTSIM_OK) return s;
    }
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_batch_project(int method, const ctsim_batch_item *items, int n, void *stream) {
    ctsim_status s = batch_check(method, items, n, true);
    if (s != CTSIM_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    // column prefix sums of every image (each plan's own scratch)
    for (int i = 0; i < n; i++) {
        const ctsim_plan *p = items[i].plan;
        if ((e = launch_prefix(items[i].in, items[i].in_dtype, p->d_xs, p->g.nx * p->g.ny, p->g.nz, p->fwd_pairs, p->g.xstride,
                               st)) != cudaSuccess)
            return cuda_fail(e, "prefix kernel");
    }
    // one persistent launch per launch-shape class (row threads, candidate groups, prefix
    // layout: 0 plain, 1 pairs, 2 staged, with the staged slots)
    std::map<std::vector<int>, std::vector<int>> classes;  // (row threads, groups, layout, FP32 out, slots)
    for (int i = 0; i < n; i++) {
        const ctsim_plan *p = items[i].plan;
        const bool staged = p->fwd_staged && !p->fwd_pairs;
        classes[{p->fwd_rows, p->fwd_groups, p->fwd_pairs ? 1 : staged ? 2 : 0,
                 items[i].out_dtype == CTSIM_F32 ? 0 : 1, staged ? p->fwd_slots : 0}].push_back(i);
    }
    for (auto &cl : classes) {
        const std::vector<int> &idx = cl.second;
        for (size_t c0 = 0; c0 < idx.size(); c0 += kBatchMax) {
            ProjBatch b;
            b.n = 0;
            b.total = 0;
            size_t smem = 0;
            for (size_t c = c0; c < std::min(idx.size(), c0 + kBatchMax); c++) {
                const ctsim_batch_item &it = items[idx[c]];
                const ctsim_plan *p = it.plan;
                ProjTask &T = b.t[b.n++];
                T.g = p->g;
                T.views = p->d_views;
                T.xs = p->d_xs;
                T.ampv = p->d_ampv;
                T.map = p->d_map;
                T.proj = it.out;
                T.out_dtype = it.out_dtype;
                T.vb = it.view_begin;
                T.vs = it.view_stride;
                T.vc = it.view_count;
                T.gx = (p->g.nu + proj_group_width() - 1) / proj_group_width();
                T.first = b.total;
                T.margin = p->margin;
                T.err = p->d_err;
                b.total += proj_task_blocks(p->g, it.view_count);
                smem = std::max(smem, cl.first[2] == 2 ? proj_staged_smem_bytes(p->g.nv, p->g.nx, p->g.ny, p->g.xstride,
                                                                                p->fwd_groups, p->fwd_rows,
                                                                                p->fwd_slots)
                                                       : proj_smem_bytes(p->g.nv, p->g.nx, p->g.ny, p->fwd_groups,
                                                                         p->fwd_rows));
            }
            const int m = method == CTSIM_PROJ_DD ? kDD : kTF;
            e = cl.first[2] == 2 ? launch_proj_staged_batch(m, cl.first[1], cl.first[0], cl.first[4], cl.first[3] != 0,
                                                            smem, b, st)
                                 : launch_proj_batch(m, cl.first[1], cl.first[0], cl.first[2] == 1, cl.first[3] != 0,
                                                     smem, b, st);
            if (e != cudaSuccess) return cuda_fail(e, "batched forward projection");
        }
    }
    return CTSIM_OK;
}

extern "C" ctsim_status ctsim_batch_backproject(int method, const ctsim_batch_item *items, int n, void *stream) {
    const bool scaled_in = (method & CTSIM_INPUT_SCALED) != 0;
    method &= ~CTSIM_INPUT_SCALED;
    ctsim_status s = batch_check(method, items, n, false);
    if (s != CTSIM_OK || n == 0) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const bool dd = method == CTSIM_BACK_DD;
    cudaError_t e;
    // each item's source: BF16/FP16 and scaled FP32 sinograms as they are, unscaled FP32
    // ones times ampv into the plan's scratch
    std::vector<const void *> src(n);
    std::vector<int> kind(n);
    for (int i = 0; i < n; i++) {
        ctsim_plan *p = items[i].plan;
        const int dt = items[i].in_dtype;
        if (scaled_in && dt != CTSIM_F32) return fail(CTSIM_ERR_ARGUMENT, "CTSIM_INPUT_SCALED takes FP32 sinograms");
        src[i] = items[i].in;
        kind[i] = dt == CTSIM_BF16 ? kSrcBF16 : dt == CTSIM_F16 ? kSrcF16 : kSrcScaled;
        if (dt == CTSIM_F32 && !scaled_in) {
            if ((s = ensure_scratch(p, st)) != CTSIM_OK) return s;
            const size_t nuv = (size_t)p->g.nu * p->g.nv;
            if ((e = launch_prescale(items[i].in, dt, p->d_ampv, p->d_ps, nuv, nuv * items[i].view_count, st)) !=
                cudaSuccess)
                return cuda_fail(e, "prescale kernel");
            src[i] = p->d_ps;
        }
    }
    // An item of at least four waves of the single-plan kernel gains nothing from sharing a
    // launch and runs on that kernel (64 registers, four blocks per SM, against up to 128
    // registers in the batched one, whose task table is indexed at run time); the same
    // block body computes every voxel, so the images do not change.
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, items[0].plan->device);
    const int large = 4 * 4 * sms;
    // classes: (z blocks per lane, float4 rows, FP32 out, source form)
    std::map<std::vector<int>, std::vector<int>> classes;
    for (int i = 0; i < n; i++) {
        const ctsim_batch_item &it = items[i];
        const ctsim_plan *p = it.plan;
        if (back_task_blocks(p->g) >= large) {
            if ((e = launch_back(dd ? kDD : kTF, dd ? p->back_mz : p->back_mz_tf, p->g, p->d_views, src[i], p->d_map,
                                 it.out, it.out_dtype, it.view_begin, it.view_stride, it.view_count, it.scale,
                                 dd ? p->back_qcap : p->back_qcap_tf, p->d_err, st, false, 0, -1, kind[i],
                                 p->d_ampv)) != cudaSuccess)
                return cuda_fail(e, "backprojection kernel");
            continue;
        }
        const size_t align = kind[i] == kSrcScaled ? 16 : 8;
        const bool vec = (p->g.nv % 4) == 0 && (reinterpret_cast<uintptr_t>(src[i]) % align) == 0;
        classes[{dd ? p->back_mz : p->back_mz_tf, vec ? 1 : 0, it.out_dtype == CTSIM_F32 ? 0 : 1, kind[i]}].push_back(i);
    }
    for (auto &cl : classes) {
        const std::vector<int> &idx = cl.second;
        for (size_t c0 = 0; c0 < idx.size(); c0 += kBatchMax) {
            BackBatch b;
            b.n = 0;
            b.total = 0;
            int qcap = 0;
            for (size_t c = c0; c < std::min(idx.size(), c0 + kBatchMax); c++) {
                const ctsim_batch_item &it = items[idx[c]];
                const ctsim_plan *p = it.plan;
                BackTask &T = b.t[b.n++];
                T.g = p->g;
                T.views = p->d_views;
                T.ps = src[idx[c]];
                T.ampv = p->d_ampv;
                T.map = p->d_map;
                T.image = it.out;
                T.out_dtype = it.out_dtype;
                T.err = p->d_err;
                T.vb = it.view_begin;
                T.vs = it.view_stride;
                T.vc = it.view_count;
                T.qcap = dd ? p->back_qcap : p->back_qcap_tf;
                T.first = b.total;
                T.scale = it.scale;
                b.total += back_task_blocks(p->g);
                qcap = std::max(qcap, T.qcap);
            }
            if ((e = launch_back_batch(dd ? kDD : kTF, cl.first[0], cl.first[1] != 0, cl.first[2] != 0,
                                       back_smem_bytes(qcap), b, st, cl.first[3])) != cudaSuccess)
                return cuda_fail(e, "batched backprojection");
        }
    }
    return CTSIM_OK;
}
