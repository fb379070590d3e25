// Matched distance-driven backprojection that allocates no memory.
//
// For callers that may not call cudaMalloc themselves or through a library: host
// frameworks that own all device memory through their own pool (MATLAB's
// gpuArray, a serving process with a fixed memory budget), or real-time loops
// where an allocation's implicit synchronisation is not acceptable.  The caller
// passes device pointers for the sinogram and the image and host pointers for
// the geometry; the per-view table, the detector amplitude table and the map
// are built on the device in one fixed, file-scope scratch array.
#include <atomic>
#include <cmath>
#include <cstring>

#include "../../include/ctsim_b200.h"
#include "kernels.cuh"

using namespace ctsim;

namespace {

// Scratch shared by every call on a device: 8 MiB, held by each GPU that loads
// the library until the process exits.
constexpr size_t kScratchBytes = (size_t)8 << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
// Device address of g_scratch, per device.  Threads that make their first call on a
// device at the same time all look up and store the same address.
std::atomic<void *> g_scratch_ptr[kMaxDevices] = {};

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Per-view table and detector amplitudes computed on the device from the
// reference's formulas (geom/cbct/cbct_proj.c:256-265, :432-450).  sin/cos are
// the device's double-precision functions; the float results agree with the
// host-built tables of the plan API to within one float rounding.
__global__ void tables_kernel(Geom g, int noviews, float dz, float oz, float dx, float dy, const double *betas,
                              const float *couchz, View *views, float *ampv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < noviews) {
        View v;
        v.sin_a = (float)sin(betas[i]);
        v.cos_a = (float)cos(betas[i]);
        const float cz = __fdiv_rn(couchz[i], dz);
        v.wz = (float)__dadd_rn(__dadd_rn(-((double)g.nz - 1.0) / 2.0, (double)oz), (double)cz);
        v.dx_sin_2 = __fmul_rn(dx, v.sin_a) * 0.5f;
        v.dx_cos_2 = __fmul_rn(dx, v.cos_a) * 0.5f;
        v.dy_sin_2 = __fmul_rn(dy, v.sin_a) * 0.5f;
        v.n_dy_cos_2 = __fmul_rn(-dy, v.cos_a) * 0.5f;
        v.couch_pd = (float)(int)couchz[i];
        views[i] = v;
    }
    const size_t nuv = (size_t)g.nu * g.nv;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < nuv; p += (size_t)gridDim.x * blockDim.x) {
        const int iu = (int)(p / g.nv), iv = (int)(p % g.nv);
        const float u = __fmul_rn(__fadd_rn((float)iu, g.wu), g.du);
        const float uu = __fadd_rn(__fmul_rn(g.sdd, g.sdd), __fmul_rn(u, u));
        const float v = __fmul_rn(__fadd_rn((float)iv, g.wv), g.dv);
        float a;
        if (g.det == 1) a = __fsqrt_rn(__fdiv_rn(__fadd_rn(uu, __fmul_rn(v, v)), uu));
        else a = (float)__ddiv_rn(__dsqrt_rn((double)__fadd_rn(__fmul_rn(g.sdd, g.sdd), __fmul_rn(v, v))), (double)g.sdd);
        ampv[p] = a;
    }
}

}  // namespace

// Implemented in capi.cu: sets the thread's last-error message.
extern ctsim_status ctsim_set_last_error(ctsim_status s, const char *msg);

extern "C" ctsim_status ctsim_back_dd_noalloc(const ctsim_geom *geom, const double *betas, const float *couchz,
                                              const bool *map, const float *d_proj, float *d_image, void *stream) {
    if (!geom || !betas || !couchz || !d_proj || !d_image)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "null argument");
    const ctsim_geom G = *geom;
    if (G.nx < 1 || G.ny < 1 || G.nz < 1 || G.nu < 2 || G.nv < 2 || G.noviews < 1)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "sizes must be positive (nu, nv >= 2)");
    if (!(G.dx > 0 && G.dy > 0 && G.dz > 0 && G.du > 0 && G.dv > 0 && G.sad > 0 && G.sdd > 0))
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "spacings and distances must be positive");
    if (G.detector_type != 0 && G.detector_type != 1)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT, "detector_type must be 1 (flat) or 0 (curved)");
    const size_t nxy = (size_t)G.nx * G.ny;
    // scratch layout: [error flag][views][betas][couchz][ampv][map]
    const size_t off_views = 256;
    const size_t off_betas = off_views + align256(sizeof(View) * G.noviews);
    const size_t off_couch = off_betas + align256(sizeof(double) * G.noviews);
    const size_t off_ampv = off_couch + align256(sizeof(float) * G.noviews);
    const size_t off_map = off_ampv + align256(sizeof(float) * (size_t)G.nu * G.nv);
    const size_t need = off_map + align256(nxy);
    if (need > kScratchBytes)
        return ctsim_set_last_error(CTSIM_ERR_ARGUMENT,
                                    "geometry too large for ctsim_back_dd_noalloc: views, detector amplitude table "
                                    "and map must fit its 8 MiB scratch (use the plan API)");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_NO_DEVICE, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return ctsim_set_last_error(CTSIM_ERR_NO_DEVICE, "device index out of range");
    void *scratch = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        // once per device, with that device current: the host-side symbol is a stand-in,
        // the kernels need the device address
        e = cudaGetSymbolAddress(&scratch, g_scratch);
        if (e != cudaSuccess || !scratch)
            return ctsim_set_last_error(CTSIM_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed");
        g_scratch_ptr[dev].store(scratch, std::memory_order_release);
    }
    unsigned char *base = static_cast<unsigned char *>(scratch);
    int *err = reinterpret_cast<int *>(base);
    View *views = reinterpret_cast<View *>(base + off_views);
    double *dbetas = reinterpret_cast<double *>(base + off_betas);
    float *dcouch = reinterpret_cast<float *>(base + off_couch);
    float *ampv = reinterpret_cast<float *>(base + off_ampv);
    uint8_t *dmap = base + off_map;

    // geometry scalars (host, no allocation), as the plan API derives them
    Geom g{};
    auto centre = [](int n, float off) { return (float)(-((double)n - 1.0) / 2.0 + (double)off); };
    g.nx = G.nx; g.ny = G.ny; g.nz = G.nz; g.nu = G.nu; g.nv = G.nv; g.det = G.detector_type;
    g.dx = G.dx; g.dy = G.dy; g.dz = G.dz; g.sad = G.sad; g.sdd = G.sdd; g.du = G.du; g.dv = G.dv;
    g.wx = centre(G.nx, G.offset_x);
    g.wy = centre(G.ny, G.offset_y);
    g.wu = centre(G.nu, G.offset_u);
    g.wv = centre(G.nv, G.offset_v);
    g.sdd_du = G.sdd / G.du;
    g.dz_dv = G.dz / G.dv;
    g.xstride = prefix_stride(G.nz);
    double rmax = 0.0;
    for (int cx = 0; cx < 2; cx++)
        for (int cy = 0; cy < 2; cy++) {
            const double xc = ((cx ? G.nx - 1 : 0) + (double)g.wx) * G.dx;
            const double yc = ((cy ? G.ny - 1 : 0) + (double)g.wy) * G.dy;
            rmax = std::fmax(rmax, std::sqrt(xc * xc + yc * yc));
        }
    const double diag = std::sqrt((double)G.dx * G.dx + (double)G.dy * G.dy);
    if (!((double)G.sad - rmax - diag > 0.0))
        return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "the source orbit must lie outside the volume");
    const double zinc_max = (double)G.dz / G.dv * G.sdd / ((double)G.sad - rmax) * 1.0001 + 1e-6;
    if (zinc_max > 9.0)
        return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED, "axial footprints wider than 10 detector rows");
    int mz = 1;
    while (mz < 8 && 32 * mz < G.nz) mz <<= 1;
    int qcap = 0;
    for (;; mz >>= 1) {
        const int rows = (int)std::fmin((double)G.nv, std::ceil(32.0 * mz * zinc_max) + 2) + 4;
        qcap = (rows + 127) / 128 * 128;
        if (back_smem_bytes(qcap) <= 200 * 1024 || mz == 1) break;
    }

    cudaStream_t st = (cudaStream_t)stream;
    // every call rewrites the whole tables; the error flag must start at zero
    if ((e = cudaMemsetAsync(err, 0, sizeof(int), st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dbetas, betas, sizeof(double) * G.noviews, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dcouch, couchz, sizeof(float) * G.noviews, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    if (map) e = cudaMemcpyAsync(dmap, map, nxy, cudaMemcpyHostToDevice, st);  // bool is one byte
    else e = cudaMemsetAsync(dmap, 1, nxy, st);
    if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    const int tb = 256;
    const int tgrid = (int)std::fmin(148.0 * 8, std::ceil(std::fmax((double)G.noviews, (double)G.nu * G.nv / 8.0) / tb));
    tables_kernel<<<tgrid, tb, 0, st>>>(g, G.noviews, G.dz, G.offset_z, G.dx, G.dy, dbetas, dcouch, views, ampv);
    if ((e = cudaGetLastError()) != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    e = launch_back_unscaled(mz, g, views, d_proj, ampv, dmap, d_image, G.noviews, qcap, err, st);
    if (e != cudaSuccess) return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    // The kernel sets the flag when a voxel column's detector rows exceed its row buffer
    // (sized from the largest axial footprint, so never for an accepted geometry); the
    // image would then be incomplete.  Reading it back waits for the backprojection.
    int flag = 0;
    if ((e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return ctsim_set_last_error(CTSIM_ERR_CUDA, cudaGetErrorString(e));
    if (flag)
        return ctsim_set_last_error(CTSIM_ERR_UNSUPPORTED,
                                    "a voxel column's detector rows exceeded the backprojection's row buffer");
    return CTSIM_OK;
}
