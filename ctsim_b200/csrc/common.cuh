// Shared device code: geometry tables and the per-column footprint math.
//
// Every footprint quantity that decides an index (umin/umax, tau, vstart, zinc,
// the FDK detector coordinates) is evaluated with explicit round-to-nearest
// intrinsics in the reference's operand order, so that it is bit-identical to
// the reference's float C (geom/cbct/cbct_proj.c, geom/cbct/cbct_back.c) and no
// multiply-add is contracted.  Accumulations elsewhere are free to use FMA.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace ctsim {

// Storage types of volumes and sinograms (all arithmetic is FP32): CTSIM_F32 = 0,
// CTSIM_BF16 = 1, CTSIM_F16 = 2 in the C ABI.
enum DType { kF32 = 0, kBF16 = 1, kF16 = 2 };

__device__ __forceinline__ float load_as_float(const void *p, size_t i, int dtype) {
    if (dtype == kBF16) return __bfloat162float(static_cast<const __nv_bfloat16 *>(p)[i]);
    if (dtype == kF16) return __half2float(static_cast<const __half *>(p)[i]);
    return static_cast<const float *>(p)[i];
}

__device__ __forceinline__ void store_from_float(void *p, size_t i, float v, int dtype) {
    if (dtype == kBF16) static_cast<__nv_bfloat16 *>(p)[i] = __float2bfloat16_rn(v);
    else if (dtype == kF16) static_cast<__half *>(p)[i] = __float2half_rn(v);
    else static_cast<float *>(p)[i] = v;
}

enum Method { kDD = 0, kTF = 1 };

constexpr int kMaxBinsDD = 16;  // iumax <= iumin + 15        geom/cbct/cbct_proj.c:343
constexpr int kMaxBinsTF = 10;  // iumax <= iumin + 9 (10)    geom/cbct/cbct_proj.c:210,612
constexpr int kMaxRowsV = 10;   // ivmax <= ivmin + 9 (10)    geom/cbct/cbct_proj.c:211,395

// Scalars shared by every kernel (passed by value).
struct Geom {
    int nx, ny, nz, nu, nv, det;  // det: 1 flat, 0 curved, 2 arc about the axis (DD pair only)
    float dx, dy, dz, sad, sdd, du, dv;
    float wx, wy, wu, wv;         // centre offsets, geom/cbct/cbct_proj.c:244-247
    float sdd_du;                 // sdd / du                  :248
    float dz_dv;                  // dz / dv (first factor of zinc, :361)
    float wz_pd;                  // -(nz-1)/2 + offset_z, geom/cbct/cbct_back.c:47
    float roff;                   // curved FDK: offset_u*du*sad/sdd, cbct_back.c:80
    float roff_var;               // curved back,var: offset_u*sad/sdd, cbct_back_var.c:70
    // FDK boundary tests "u < 1E-6 || u > nu - 1 - 1E-6" are done in double in the
    // reference (cbct_back.c:90, :105-111); these are the exact float thresholds:
    // u < 1e-6 (double) <=> u < u_lo ; u > nu-1-1e-6 (double) <=> u > u_hi (floats).
    float u_lo, u_hi, v_lo, v_hi;
    float v_clamp_lo, v_clamp_hi; // hpd clamps 0.5 and nv - 1.5 as floats (cbct_back.c:110-111)
    float rdv;                    // RN(1/dv) for the correctly rounded division by dv, 0 = use IEEE division
    float add, sad_add;           // arc detector: radius ADD, sad / add (geom/cbct/cbct_proj3.c:337-355)
    int xstride;                  // column stride (floats) of the plain prefix-sum layout: prefix_stride(nz)
};

// Column stride of the plain prefix-sum layout: X[0..nz] and at least one copy of X[nz]
// above it, rounded up to 4 floats so that every column starts on a 16-byte boundary
// (the bulk copies of the staged forward projector need that).
__host__ __device__ inline int prefix_stride(int nz) { return (nz + 2 + 3) & ~3; }

// Per-view constants, geom/cbct/cbct_proj.c:256-265 and cbct_back.c:50-52.
struct View {
    float sin_a, cos_a;  // (float) sin/cos of the double angle
    float wz;            // axial centre incl. couch shift / dz
    float dx_sin_2, dx_cos_2, dy_sin_2, n_dy_cos_2;
    float couch_pd;      // (float)(int) couchz, the FDK couch shift truncated to int
};

// Exact float / double operations (no contraction).
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// floor() of x in [0, 2^23) without conversion instructions (which run on the
// narrow XU pipe): x + 2^23 rounded toward -inf has ulp 1, so its bit pattern is
// 0x4B000000 + floor(x).  Returns the integer; *fl receives floor(x) as a float.
constexpr float kTwo23 = 8388608.0f;
__device__ __forceinline__ int floor_pos(float x, float *fl) {
    const float t = __fadd_rd(x, kTwo23);
    *fl = __fsub_rn(t, kTwo23);
    return __float_as_int(t) - 0x4B000000;
}
__device__ __forceinline__ int floor_pos(float x) { return __float_as_int(__fadd_rd(x, kTwo23)) - 0x4B000000; }
// (float)i for 0 <= i < 2^23, exact, without a conversion instruction.
__device__ __forceinline__ float small_int_to_float(int i) { return __fsub_rn(__int_as_float(i + 0x4B000000), kTwo23); }

// Correctly rounded a / d given r = RN(1/d) (Markstein): q = RN(a r), e = a - q d
// (exact by FMA), RN(q + e r).  Valid when d's significand is not all ones and no
// overflow/underflow occurs -- the host checks d and otherwise passes r = 0, which
// selects the IEEE division.
__device__ __forceinline__ float div_by(float a, float d, float r) {
    if (r == 0.0f) return __fdiv_rn(a, d);
    const float q = __fmul_rn(a, r);
    const float e = __fmaf_rn(-q, d, a);
    return __fmaf_rn(e, r, q);
}

// Footprint of one voxel column in one view.
struct ColumnFP {
    float ampu;    // in-plane amplitude dx / max(|cos phi|, |sin phi|) / 10
    float zinc;    // voxel height in detector rows
    float vstart;  // detector row (before +0.5) of the bottom edge of voxel 0
    float p0, p1, p2, p3;  // DD: p0 = umin', p1 = umax' (shifted, clamped); TF: tau[0..3] (sorted, unshifted)
    int iumin, iumax;
    bool hit;
};

// Detector coordinate of the ray through (num, den) in the rotated frame
// (geom/cbct/cbct_proj.c:301 flat, :316 curved).
__device__ __forceinline__ float u_of(const Geom &g, float num, float den) {
    if (g.det == 1) return fsub(fdiv(fmul(g.sdd_du, num), den), g.wu);
    if (g.det == 2) {
        // arc: fan angle gam, arc angle xi = gam + asin(sad/add sin gam) where the ray meets
        // the arc, u = xi * add / du - wu (geom/cbct/cbct_proj3.c:337-343)
        const float gam = (float)atan((double)fdiv(num, den));
        const float xi = (float)__dadd_rn((double)gam, asin(__dmul_rn((double)g.sad_add, sin((double)gam))));
        return fsub(fdiv(fmul(xi, g.add), g.du), g.wu);
    }
    double r = (double)fdiv(num, den);
    return (float)__dsub_rn(__dmul_rn((double)g.sdd_du, atan(r)), (double)g.wu);
}

// Exact transcription of the per-column footprint (DD: cbct_proj.c:282-372,
// TF: cbct_proj.c:531-656).
template <int METHOD>
__device__ __forceinline__ ColumnFP column_footprint(const Geom &g, const View &v, int ix, int iy) {
    ColumnFP c;
    c.hit = false;
    float xc = fmul(fadd((float)ix, g.wx), g.dx);
    float yc = fmul(fadd((float)iy, g.wy), g.dy);
    float tproj0 = fsub(fmul(xc, v.cos_a), fmul(yc, v.sin_a));
    float dsxy0 = fadd(fadd(g.sad, fmul(xc, v.sin_a)), fmul(yc, v.cos_a));
    float r = __fsqrt_rn(fadd(fmul(tproj0, tproj0), fmul(dsxy0, dsxy0)));
    float cos_gamma = fdiv(dsxy0, r);
    float sin_gamma = fdiv(tproj0, r);
    float cos_phi = fabsf(fsub(fmul(v.cos_a, cos_gamma), fmul(v.sin_a, sin_gamma)));
    float sin_phi = fabsf(fadd(fmul(v.sin_a, cos_gamma), fmul(v.cos_a, sin_gamma)));
    float umin, umax;
    int maxbins;
    if (METHOD == kDD) {
        if (cos_phi > sin_phi) {
            c.ampu = fdiv(fdiv(g.dx, cos_phi), 10.0f);
            umin = u_of(g, fadd(tproj0, v.dx_cos_2), fadd(dsxy0, v.dx_sin_2));
            umax = u_of(g, fsub(tproj0, v.dx_cos_2), fsub(dsxy0, v.dx_sin_2));
        } else {
            c.ampu = fdiv(fdiv(g.dx, sin_phi), 10.0f);
            umin = u_of(g, fadd(tproj0, v.dy_sin_2), fadd(dsxy0, v.n_dy_cos_2));
            // the arc code takes this edge from the x offsets (cbct_proj3.c:352, cbct_back3.c:299)
            umax = g.det == 2 ? u_of(g, fsub(tproj0, v.dx_cos_2), fsub(dsxy0, v.dx_sin_2))
                              : u_of(g, fsub(tproj0, v.dy_sin_2), fsub(dsxy0, v.n_dy_cos_2));
        }
        if (umin >= umax) { float t = umax; umax = umin; umin = t; }
        maxbins = kMaxBinsDD;
    } else {
        c.ampu = fdiv(fdiv(g.dx, cos_phi > sin_phi ? cos_phi : sin_phi), 10.0f);
        float t0 = u_of(g, fadd(fadd(tproj0, v.dx_cos_2), v.dy_sin_2), fadd(fadd(dsxy0, v.dx_sin_2), v.n_dy_cos_2));
        float t1 = u_of(g, fadd(fsub(tproj0, v.dx_cos_2), v.dy_sin_2), fadd(fsub(dsxy0, v.dx_sin_2), v.n_dy_cos_2));
        float t2 = u_of(g, fsub(fadd(tproj0, v.dx_cos_2), v.dy_sin_2), fsub(fadd(dsxy0, v.dx_sin_2), v.n_dy_cos_2));
        float t3 = u_of(g, fsub(fsub(tproj0, v.dx_cos_2), v.dy_sin_2), fsub(fsub(dsxy0, v.dx_sin_2), v.n_dy_cos_2));
        // sorting network (0,1) (2,3) (0,2) (1,3) (1,2), cbct_proj.c:569-599
        float t;
        if (t0 > t1) { t = t0; t0 = t1; t1 = t; }
        if (t2 > t3) { t = t2; t2 = t3; t3 = t; }
        if (t0 > t2) { t = t0; t0 = t2; t2 = t; }
        if (t1 > t3) { t = t1; t1 = t3; t3 = t; }
        if (t1 > t2) { t = t1; t1 = t2; t2 = t; }
        c.p0 = t0; c.p1 = t1; c.p2 = t2; c.p3 = t3;
        umin = t0;
        umax = t3;
        maxbins = kMaxBinsTF;
    }
    umin = fadd(umin, 0.5f);
    if (!(umin > 0.0f)) umin = 0.0f;
    umax = fadd(umax, 0.5f);
    if (!(umax < (float)g.nu)) umax = (float)g.nu;
    if (umin > umax) return c;
    int lo = (int)floorf(umin), hi = (int)floorf(umax);
    hi = min(hi, g.nu - 1);
    hi = min(hi, lo + maxbins - 1);
    c.iumin = lo;
    c.iumax = hi;
    if (METHOD == kDD) { c.p0 = umin; c.p1 = umax; }
    // axial footprint, cbct_proj.c:361-372
    c.zinc = fdiv(fmul(g.dz_dv, g.sdd), dsxy0);
    c.vstart = (float)__dsub_rn(__dmul_rn(__dsub_rn((double)v.wz, 0.5), (double)c.zinc), (double)g.wv);
    int s = (int)floorf(fdiv(fsub(-1.0f, c.vstart), c.zinc));
    int e = (int)ceilf(fdiv(fsub((float)(g.nv + 1), c.vstart), c.zinc));
    s = max(s, 0);
    e = min(e, g.nz);
    c.hit = (s <= e);
    return c;
}

// u weight of detector column iu for a footprint (DD: cbct_proj.c:346-359,
// TF: trapezoid integral cbct_proj.c:614-643).
template <int METHOD>
__device__ __forceinline__ float u_weight(int iu, int iumin, int iumax, float p0, float p1, float p2, float p3) {
    if (METHOD == kDD) {
        if (iumin == iumax) return fsub(p1, p0);
        if (iu == iumin) return fsub((float)(iumin + 1), p0);
        if (iu == iumax) return fsub(p1, (float)iumax);
        return 1.0f;
    } else {
        float w = 0.0f;
        float bl = (float)iu - 0.5f, br = (float)iu + 0.5f;
        float xl = bl > p0 ? bl : p0, xr = br < p1 ? br : p1;
        if (xr > xl) {
            float a = fsub(xr, p0), b = fsub(xl, p0);
            w = fadd(w, fmul(fdiv(fsub(fmul(a, a), fmul(b, b)), fsub(p1, p0)), 0.5f));  // /2 is exact
        }
        xl = bl > p1 ? bl : p1; xr = br < p2 ? br : p2;
        if (xr > xl) w = fadd(w, fsub(xr, xl));
        xl = bl > p2 ? bl : p2; xr = br < p3 ? br : p3;
        if (xr > xl) {
            float a = fsub(xl, p3), b = fsub(xr, p3);
            w = fadd(w, fmul(fdiv(fsub(fmul(a, a), fmul(b, b)), fsub(p3, p2)), 0.5f));
        }
        return w;
    }
}

// Shifted, clamped axial extent [vmin', vmax'] of voxel iz (cbct_proj.c:382-390).
__device__ __forceinline__ void voxel_v_extent(const Geom &g, float vstart, float zinc, int iz, float &vmin,
                                               float &vmax) {
    vmin = fadd(vstart, fmul((float)iz, zinc));
    vmax = fadd(vmin, zinc);
    vmin = fadd(vmin, 0.5f);
    if (!(vmin > 0.0f)) vmin = 0.0f;
    vmax = fadd(vmax, 0.5f);
    if (!(vmax < (float)g.nv)) vmax = (float)g.nv;
}

}  // namespace ctsim
