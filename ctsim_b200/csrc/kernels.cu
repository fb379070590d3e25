// Projector kernels for sm_100a.
//
//   back_kernel<METHOD,MZ>   matched backprojection A^T (distance-driven / separable footprint)
//   prefix_kernel            per-column axial prefix sums of the volume (input of A)
//   proj_kernel<METHOD>      forward projection A
//   pd_kernel<OFF,MZ>        voxel-driven bilinear FDK backprojection (back,pd / back,hpd)
//   scale_kernel             y *= s
//
// Layouts (reference MEX conventions): image[iz][iy][ix], proj[view][iu][iv].
#include "kernels.cuh"

#include <map>
#include <mutex>
#include <utility>

namespace ctsim {

constexpr unsigned kFull = 0xffffffffu;

// Rows r0 .. r0+3 of one detector column of a sinogram source (element offset off of row
// r0), times ampv at the same element for the unscaled sources.  VEC: nv a multiple of 4
// and the source aligned (one 16-byte FP32 or 8-byte 16-bit load); otherwise rows at or
// past nv read as 0.
template <int SRC, bool VEC>
__device__ __forceinline__ float4 load_rows4(const void *__restrict__ src, const float *__restrict__ ampv, size_t off,
                                             size_t aoff, int r0, int nv) {
    float4 p;
    if (SRC == kSrcScaled || SRC == kSrcF32) {
        const float *pr = static_cast<const float *>(src) + off;
        if (VEC) {
            p = __ldg(reinterpret_cast<const float4 *>(pr));
        } else {
            p.x = __ldg(pr);
            p.y = r0 + 1 < nv ? __ldg(pr + 1) : 0.f;
            p.z = r0 + 2 < nv ? __ldg(pr + 2) : 0.f;
            p.w = r0 + 3 < nv ? __ldg(pr + 3) : 0.f;
        }
    } else {
        const unsigned short *pr = static_cast<const unsigned short *>(src) + off;
        unsigned short h[4];
        if (VEC) {
            const uint2 u = __ldg(reinterpret_cast<const uint2 *>(pr));
            h[0] = (unsigned short)(u.x & 0xffffu); h[1] = (unsigned short)(u.x >> 16);
            h[2] = (unsigned short)(u.y & 0xffffu); h[3] = (unsigned short)(u.y >> 16);
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) h[i] = r0 + i < nv ? __ldg(pr + i) : (unsigned short)0;
        }
        float f[4];
#pragma unroll
        for (int i = 0; i < 4; i++)
            f[i] = SRC == kSrcBF16 ? __uint_as_float((unsigned)h[i] << 16) : __half2float(__ushort_as_half(h[i]));
        p = make_float4(f[0], f[1], f[2], f[3]);
    }
    if (SRC != kSrcScaled) {  // axial amplitude applied here instead of in a scratch copy
        const float *ar = ampv + aoff;
        float4 a;
        if (VEC) {
            a = __ldg(reinterpret_cast<const float4 *>(ar));
        } else {
            a.x = __ldg(ar);
            a.y = r0 + 1 < nv ? __ldg(ar + 1) : 0.f;
            a.z = r0 + 2 < nv ? __ldg(ar + 2) : 0.f;
            a.w = r0 + 3 < nv ? __ldg(ar + 3) : 0.f;
        }
        p.x *= a.x; p.y *= a.y; p.z *= a.z; p.w *= a.w;
    }
    return p;
}

// ---------------------------------------------------------------------------
// A^T: one warp per voxel column, lanes along z; 8 columns (consecutive ix) per block.
// For each view the warp forms, in shared memory, the u-weighted detector column
//     q[iv] = sum_iu w_u(iu) * ps[iu][iv]        (ps = proj * ampv)
// over the rows the column's voxels can touch (4 rows per lane, float4 loads).  Each
// voxel then sums q over the rows its axial extent covers with the distance-driven
// row weights of geom/cbct/cbct_back.c:318-357, its edges vmin/vmax computed with the
// reference's float operations (usually two or three rows per voxel).  The edges sit
// hundreds of rows up the detector, where one float rounding moves a voxel's weight by
// ~1e-5 of itself; evaluating them exactly as the reference does keeps each voxel's
// value within a few float roundings of the reference's instead of adding noise of
// that size.  Accumulation over views stays in registers; no atomics.
// ---------------------------------------------------------------------------
// The work of one block (8 columns of one row iy), as a device function: the plain
// kernel runs it for blockIdx.x, the batched kernel for each of its work items.
// 32-bit shared load ordered after the warp's earlier shared stores (compiler barrier).
__device__ __forceinline__ float lds_ordered(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    return v;
}

template <int METHOD, int MZ, bool VEC, int SRC, bool SUM = false>
__device__ __forceinline__ void back_block(const Geom g, const View *__restrict__ views, const void *__restrict__ ps,
                                           const uint8_t *__restrict__ map, void *__restrict__ image, int out_dtype,
                                           int view_begin, int view_stride, int view_count, float scale, int qcap,
                                           int *__restrict__ err, const float *__restrict__ ampv, float *smem,
                                           int block) {
    constexpr int kWS = 17;  // row stride of the per-warp weight table (conflict-free writes)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *wtab = smem + warp * (32 * kWS + 32 * 8 + qcap);  // [32 views][17] u weights of the view chunk
    // [32 views] per-view scalars of the chunk, written by the view's own lane:
    // {ampu, zinc, vstart, iumin | nb << 16}, {rbase | r_hi << 16, path + 1 (0: no rows), -, -}
    float4 *vtab = reinterpret_cast<float4 *>(wtab + 32 * kWS);  // 16-byte aligned: 32 * 17 * 4 = 2176
    float *Q = wtab + 32 * kWS + 32 * 8;                         // [qcap] q per row
    const int tiles_x = (g.nx + 7) >> 3;
    const int iy = block / tiles_x;
    const int ix = (block % tiles_x) * 8 + warp;
    if (ix >= g.nx || iy >= g.ny) return;
    const size_t nxy = (size_t)g.nx * g.ny;
    const size_t nuv = (size_t)g.nu * g.nv;
    const bool on = map[iy * g.nx + ix] != 0;
    const float fnv = (float)g.nv;
    const int nvm1 = g.nv - 1;
    const int zpass = 32 * MZ;
    for (int iz0 = 0; iz0 < g.nz; iz0 += zpass) {
        const int izn = min(zpass, g.nz - iz0);
        const float fz_first = (float)iz0, fz_last = (float)(iz0 + izn - 1);
        float acc[MZ];
#pragma unroll
        for (int m = 0; m < MZ; m++) acc[m] = 0.0f;
        const float fz_lane = (float)(iz0 + lane);
        if (SUM) {
            // continue the per-voxel view sum (scale 1) that the previous view chunk left in
            // the FP32 image; the sum runs in view order either way
            const float *src = static_cast<const float *>(image) + (size_t)(iz0 + lane) * nxy + (size_t)iy * g.nx + ix;
#pragma unroll
            for (int m = 0; m < MZ; m++)
                if (lane + 32 * m < izn) acc[m] = src[(size_t)(32 * m) * nxy];
        }
        if (on) {
            for (int k0 = 0; k0 < view_count; k0 += 32) {
                ColumnFP my;
                my.hit = false;
                const int kl = k0 + lane;
                if (kl < view_count) my = column_footprint<METHOD>(g, views[view_begin + kl * view_stride], ix, iy);
                // lane-parallel u weights of this lane's view (geom/cbct/cbct_back.c:288-301, :549-578)
                // A voxel's vmax - vmin is zinc within 1.5 float ulps of nv (< 2^-10 for nv <=
                // 8192), so away from zinc = 1 and 2 by a margin every voxel of the view covers
                // the same number of rows give or take one: n = k_hi - k_lo is 0 or 1 (zinc < 1)
                // or 1 or 2 (1 < zinc < 2).  Those views run branch-free (paths 1 and 2 below).
                constexpr float kMargin = 1.0f / 256.0f;
                __syncwarp();  // the previous chunk's reads of wtab and vtab are done
                {
                    int path1 = 0, rows = 0;
                    if (my.hit) {
                        const int nb = my.iumax - my.iumin + 1;
                        for (int b = 0; b < nb; b++)
                            wtab[lane * kWS + b] =
                                u_weight<METHOD>(my.iumin + b, my.iumin, my.iumax, my.p0, my.p1, my.p2, my.p3);
                        // rows reachable by voxels [iz0, iz0+izn) (the reference's clamped
                        // extents, monotone in iz)
                        const float zinc = my.zinc, vstart = my.vstart;
                        const float a0u = fadd(fadd(vstart, fmul(fz_first, zinc)), 0.5f);
                        const float b1u = fadd(fadd(fadd(vstart, fmul(fz_last, zinc)), zinc), 0.5f);
                        const float a0 = fmaxf(a0u, 0.0f), b1 = fminf(b1u, fnv);
                        if (a0 < fnv && b1 >= 0.0f) {
                            const int r_lo = floor_pos(a0);
                            int r_hi = min(floor_pos(b1), nvm1);
                            if (r_lo <= r_hi) {
                                const int rbase = r_lo & ~3;
                                // every voxel of the pass exists and lies inside the detector
                                bool inside = a0u > 0.0f && b1u < fnv && izn == zpass;
                                if (r_hi - rbase + 1 > qcap) {  // rows rbase..r_hi must fit
                                    atomicOr(err, 1);
                                    r_hi = rbase + qcap - 1;
                                    inside = false;
                                }
                                path1 = 1 + (!inside ? 0 : zinc < 1.0f - kMargin ? 1
                                                     : (zinc > 1.0f + kMargin && zinc < 2.0f - kMargin) ? 2 : 0);
                                rows = rbase | (r_hi << 16);
                            }
                        }
                        vtab[2 * lane] = make_float4(my.ampu, zinc, vstart, __int_as_float(my.iumin | (nb << 16)));
                    }
                    vtab[2 * lane + 1] = make_float4(__int_as_float(rows), __int_as_float(path1), 0.f, 0.f);
                }
                __syncwarp();
                const int nk = min(32, view_count - k0);
                for (int j = 0; j < nk; j++) {
                    const float4 pb = vtab[2 * j + 1];
                    const int path1 = __float_as_int(pb.y);
                    if (path1 == 0) continue;  // no footprint or no rows
                    const float4 pa = vtab[2 * j];
                    const float ampu = pa.x, zinc = pa.y, vstart = pa.z;
                    const int iumin = __float_as_int(pa.w) & 0xffff, nb = __float_as_int(pa.w) >> 16;
                    const int rbase = __float_as_int(pb.x) & 0xffff, r_hi = __float_as_int(pb.x) >> 16;
                    // q over rows [rbase, r_hi], 128 rows per pass (the voxels read rows
                    // [r_lo, r_hi] only)
                    const float *wj = wtab + j * kWS;
                    const size_t pv = (size_t)(k0 + j) * nuv + (size_t)iumin * g.nv;  // element offsets
                    const size_t av = (size_t)iumin * g.nv;
                    for (int c = rbase; c <= r_hi; c += 128) {
                        const int r0 = c + 4 * lane;
                        float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f;
                        if (r0 <= r_hi) {
                            for (int b = 0; b < nb; b++) {
                                const float w = wj[b];
                                const float4 p = load_rows4<SRC, VEC>(ps, ampv, pv + (size_t)b * g.nv + r0,
                                                                      av + (size_t)b * g.nv + r0, r0, g.nv);
                                q0 = fmaf(w, p.x, q0); q1 = fmaf(w, p.y, q1);
                                q2 = fmaf(w, p.z, q2); q3 = fmaf(w, p.w, q3);
                            }
                        }
                        *reinterpret_cast<float4 *>(Q + (r0 - rbase)) = make_float4(q0, q1, q2, q3);
                    }
                    __syncwarp();
                    // Each voxel: the reference's clamped extent and row weights
                    // (geom/cbct/cbct_back.c:318-357); rows [k_lo, k_hi] lie in [r_lo, r_hi]
                    // because the edges are monotone in iz.
                    const float *qb = Q - rbase;
                    // shared address of row k is qadj + 4 * bits(k + 2^23) (mod 2^32)
                    const uint32_t qadj = (uint32_t)__cvta_generic_to_shared(Q) - 4u * (uint32_t)rbase -
                                          (0x4B000000u << 2);
                    // Paths 1 and 2 always read the rows k_lo .. k_lo + 1 (+ 2) (the row buffer has 4
                    // spare floats; rows past r_hi may hold anything, so their terms are selected,
                    // never multiplied by zero).
                    const int path = path1 - 1;
                    if (path == 1) {
#pragma unroll
                        for (int m = 0; m < MZ; m++) {
                            const float izv = fz_lane + (float)(32 * m);  // exact
                            const float vpre = fadd(vstart, fmul(izv, zinc));
                            const float vmin = fadd(vpre, 0.5f);
                            const float vmax = fadd(fadd(vpre, zinc), 0.5f);
                            const float tlo = __fadd_rd(vmin, kTwo23), thi = __fadd_rd(vmax, kTwo23);
                            const uint32_t qa = qadj + (__float_as_uint(tlo) << 2);
                            const float q0 = lds_ordered(qa), q1 = lds_ordered(qa + 4u);
                            // one row: (vmax - vmin) q0; two: (k_lo + 1 - vmin) q0 + (vmax - k_hi) q1,
                            // where k_hi = k_lo + 1 (kf, exact)
                            const float one = fsub(vmax, vmin) * q0;
                            const float kf = fsub(tlo, kTwo23 - 1.0f);
                            const float two = fmaf(fsub(vmax, kf), q1, fsub(kf, vmin) * q0);
                            acc[m] = fmaf(ampu, thi == tlo ? one : two, acc[m]);
                        }
                    } else if (path == 2) {
#pragma unroll
                        for (int m = 0; m < MZ; m++) {
                            const float izv = fz_lane + (float)(32 * m);
                            const float vpre = fadd(vstart, fmul(izv, zinc));
                            const float vmin = fadd(vpre, 0.5f);
                            const float vmax = fadd(fadd(vpre, zinc), 0.5f);
                            const float tlo = __fadd_rd(vmin, kTwo23), thi = __fadd_rd(vmax, kTwo23);
                            const uint32_t qa = qadj + (__float_as_uint(tlo) << 2);
                            const float q0 = lds_ordered(qa), q1 = lds_ordered(qa + 4u), q2 = lds_ordered(qa + 8u);
                            const bool three = fsub(thi, tlo) == 2.0f;
                            const float wl = fsub(vmax, fsub(thi, kTwo23));
                            // two rows: w0 q0 + wl q1; three: w0 q0 + q1 + wl q2 (the reference's row order)
                            float vox = fmaf(three ? 1.0f : wl, q1, fsub(fsub(tlo, kTwo23 - 1.0f), vmin) * q0);
                            vox = three ? fmaf(wl, q2, vox) : vox;
                            acc[m] = fmaf(ampu, vox, acc[m]);
                        }
                    } else {
#pragma unroll
                        for (int m = 0; m < MZ; m++) {
                            const float izv = fz_lane + (float)(32 * m);  // exact
                            const float vpre = fadd(vstart, fmul(izv, zinc));                // vstart + iz * zinc
                            const float vmin = fmaxf(fadd(vpre, 0.5f), 0.0f);                 // max(vmin + 0.5, 0)
                            const float vmax = fminf(fadd(fadd(vpre, zinc), 0.5f), fnv);      // min(vmax + 0.5, nv)
                            if (izv <= fz_last && vmin <= vmax) {
                                float flo, fhi;
                                const int klo = floor_pos(vmin, &flo);
                                int khi = floor_pos(vmax, &fhi);
                                if (khi > nvm1) { khi = nvm1; fhi = fsub(fnv, 1.0f); }
                                if (khi > klo + (kMaxRowsV - 1)) {
                                    khi = klo + (kMaxRowsV - 1);
                                    fhi = fadd(flo, (float)(kMaxRowsV - 1));
                                }
                                khi = min(khi, r_hi);  // only after a row-buffer overflow (flagged above)
                                float vox = 0.0f;
                                if (klo == khi) {
                                    vox = fsub(vmax, vmin) * qb[klo];
                                } else if (klo < khi) {
                                    vox = fsub(fadd(flo, 1.0f), vmin) * qb[klo];
                                    for (int k = klo + 1; k < khi; k++) vox += qb[k];
                                    vox = fmaf(fsub(vmax, fhi), qb[khi], vox);
                                }
                                acc[m] = fmaf(ampu, vox, acc[m]);
                            }
                        }
                    }
                    __syncwarp();
                }
                __syncwarp();
            }
        }
#pragma unroll
        for (int m = 0; m < MZ; m++) {
            const int dz = lane + 32 * m;
            if (dz < izn)
                store_from_float(image, (size_t)(iz0 + dz) * nxy + (size_t)iy * g.nx + ix, on ? acc[m] * scale : 0.0f,
                                 out_dtype);
        }
    }
}

// ps = proj * ampv (the axial amplitude the reference applies to the backprojected
// view in place, geom/cbct/cbct_back.c:196-214), into scratch.
// Four resident blocks per SM (registers capped at 64): measured on B200 at config 2,
// DD 110 -> 100 ms and SF 143 -> 104 ms against the uncapped 80-118 registers.
template <int METHOD, int MZ, bool VEC, int SRC = kSrcScaled, bool SUM = false>
__global__ void __launch_bounds__(256, 4) back_kernel(Geom g, const View *__restrict__ views,
                                                   const void *__restrict__ ps, const uint8_t *__restrict__ map,
                                                   void *__restrict__ image, int out_dtype, int view_begin,
                                                   int view_stride, int view_count, float scale, int qcap,
                                                   int *__restrict__ err, const float *__restrict__ ampv,
                                                   int block_base) {
    extern __shared__ float smem[];
    back_block<METHOD, MZ, VEC, SRC, SUM>(g, views, ps, map, image, out_dtype, view_begin, view_stride,
                                                view_count, scale, qcap, err, ampv, smem, block_base + blockIdx.x);
}

__global__ void prescale_kernel(const void *__restrict__ proj, int in_dtype, const float *__restrict__ ampv,
                                float *__restrict__ ps, size_t nuv, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        ps[i] = load_as_float(proj, i, in_dtype) * (ampv ? ampv[i % nuv] : 1.0f);
}

// ---------------------------------------------------------------------------
// Axial prefix sums of every voxel column (input of the forward projector),
// X[k] = sum_{j<k} image[j][col], k = 0..nz, col = iy*nx + ix, in one of two layouts:
// * PAIRS: xc[col][k] = (X[k], X[k+1] - X[k]) as float2, with the top pair (X[nz], 0), so
//   X(s) = X[k] + (s - k) * slope is one aligned 8-byte load and one FMA for 0 <= s <= nz;
// * single: xc[col][k] = X[k] as float (half the bytes: better when the volume's prefix
//   does not stay cache-resident; measured on B200 at 512^2 x 256), columns xstride =
//   prefix_stride(nz) floats apart, with X[nz] repeated above X[nz] up to the stride.
// 32 columns per block; a 32x32 tile is transposed through shared memory so that the
// image reads and the prefix writes are coalesced.
// ---------------------------------------------------------------------------
template <bool PAIRS>
__global__ void __launch_bounds__(256) prefix_kernel(const void *__restrict__ image, int in_dtype,
                                                     float *__restrict__ xs, int nxy, int nz, int xstride) {
    __shared__ float tile[32][33];
    __shared__ float carry[32];
    const int c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    const size_t stride = PAIRS ? (size_t)nz + 1 : (size_t)xstride;
    if (threadIdx.x < 32) carry[threadIdx.x] = 0.0f;
    for (int z0 = 0; z0 < nz; z0 += 32) {
        __syncthreads();
        for (int zz = ty; zz < 32; zz += 8) {
            const int z = z0 + zz, c = c0 + tx;
            tile[zz][tx] = (z < nz && c < nxy) ? load_as_float(image, (size_t)z * nxy + c, in_dtype) : 0.0f;
        }
        __syncthreads();
        // warp ty scans columns ty, ty+8, ty+16, ty+24 along z (lane = z)
        for (int cc = ty; cc < 32; cc += 8) {
            float v = tile[tx][cc];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float n = __shfl_up_sync(kFull, v, o);
                if (tx >= o) v += n;
            }
            const float base = carry[cc];
            const float xtop = base + v;                        // X[z + 1]
            const float xprev = __shfl_up_sync(kFull, xtop, 1);  // X[z] from the lane below
            const float xbot = tx == 0 ? base : xprev;
            const int c = c0 + cc, z = z0 + tx;
            if (c < nxy && z < nz) {
                if (PAIRS) reinterpret_cast<float2 *>(xs)[(size_t)c * stride + z] = make_float2(xbot, xtop - xbot);
                else xs[(size_t)c * stride + z + 1] = xtop;
            }
            const float tot = __shfl_sync(kFull, v, 31);
            __syncwarp();
            if (tx == 0) carry[cc] = base + tot;
        }
    }
    __syncthreads();
    if (threadIdx.x < 32 && c0 + threadIdx.x < nxy) {
        const size_t c = c0 + threadIdx.x;
        if (PAIRS) {
            reinterpret_cast<float2 *>(xs)[c * stride + nz] = make_float2(carry[threadIdx.x], 0.0f);
        } else {
            xs[c * stride] = 0.0f;
            for (size_t k = nz + 1; k < stride; k++) xs[c * stride + k] = carry[threadIdx.x];
        }
    }
}

constexpr int kTU = 8;
constexpr int kProjMaxThreads = 256;
constexpr int kMaxLines = 2048;

// X(s): integral of a voxel column from its bottom edge to axial position s (in
// voxels, already clamped to [0, nz]) from the column's prefix (x: its first entry).
template <bool PAIRS>
__device__ __forceinline__ float column_integral(const float *__restrict__ x, float s, int nzm1, float fnzm1) {
    float fl;
    int k = floor_pos(s, &fl);
    if (PAIRS) {
        const float2 p = __ldg(reinterpret_cast<const float2 *>(x) + k);
        return fmaf(s - fl, p.y, p.x);
    }
    if (k > nzm1) { k = nzm1; fl = fnzm1; }
    const float a = __ldg(x + k), b = __ldg(x + k + 1);
    return fmaf(s - fl, b - a, a);
}

// Dynamic shared-memory layout of proj_kernel.
// groups: candidate-parallel thread groups, each with its own accumulator copy.
struct ProjSmem {
    int nq, nt, nlines, groups;
    __host__ __device__ size_t acc_bytes() const { return (size_t)groups * kTU * nq * 16; }
    __host__ __device__ size_t bytes() const {
        return acc_bytes() + (size_t)nt * (6 + kTU) * 4 + (size_t)(2 * nlines + 1 + 32) * 4;
    }
};

// A: one block per (group of kTU detector columns, view).  Candidate voxel columns
// are enumerated line by line (lines across the ray direction; the projected column
// centre is monotone along a line, so a line's candidates form one interval found by
// binary search).  Each candidate's footprint is evaluated exactly.  Thread t owns
// detector rows 4t..4t+3 and adds, for every candidate hitting its group,
//     w_u(iu) * ampu * zinc * (X(iv+1) - X(iv))
// -- the integral form of the distance-driven axial weights
// (geom/cbct/cbct_proj.c:382-420) -- into float4 shared-memory accumulators that only
// it touches: no atomics, deterministic.  A block of NT threads holds NT / R groups
// of R row threads (R a multiple of 32, passed by the launcher): group g takes candidates
// g, g + groups, ... into its own accumulators, summed in group order at the store,
// so short detectors (few rows) still keep 8 warps busy per block.
template <int METHOD, int GROUPS, bool PAIRS>
__device__ __forceinline__ void proj_block(const Geom g, const View *__restrict__ views, const float *__restrict__ xs,
                                           const float *__restrict__ ampv, const uint8_t *__restrict__ map,
                                           void *__restrict__ proj, int out_dtype, int view_begin, int view_stride,
                                           float margin, float4 *acc4, int bx, int by) {
    // acc4: [GROUPS][kTU][nq] row quads, then the arrays below (dynamic shared memory)
    const int NT = blockDim.x;
    constexpr int groups = GROUPS;
    const int R = NT / GROUPS;
    const int nq0 = (g.nv + 3) >> 2;
    const int nlines0 = max(g.nx, g.ny);
    int *s_col = reinterpret_cast<int *>(acc4 + groups * kTU * nq0);
    float *s_b0 = reinterpret_cast<float *>(s_col + NT);
    float *s_iz = s_b0 + NT;
    int *s_rlo = reinterpret_cast<int *>(s_iz + NT);
    int *s_rhi = s_rlo + NT;
    int *s_j = s_rhi + NT;
    float *s_wf = reinterpret_cast<float *>(s_j + NT);  // [NT][kTU]
    int *line_start = reinterpret_cast<int *>(s_wf + NT * kTU);
    int *line_off = line_start + nlines0;
    int *s_warp_tot = line_off + nlines0 + 1;

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int grp = GROUPS == 1 ? 0 : t / R;  // candidate group
    const int gwarp = GROUPS == 1 ? warp : (t - grp * R) >> 5;  // warp within the group
    const int iu0 = bx * kTU;
    const int k = by;
    const View v = views[view_begin + k * view_stride];
    const int nv = g.nv;
    const int nq = (nv + 3) >> 2;
    for (int i = t; i < groups * kTU * nq; i += NT) acc4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 *gacc = acc4 + grp * kTU * nq;

    // lines of constant iy when the rays run mostly along y, else lines of constant ix
    const bool rows = fabsf(v.cos_a) >= fabsf(v.sin_a);
    const int nlines = rows ? g.ny : g.nx;
    const int npos = rows ? g.nx : g.ny;
    const float ulo = (float)iu0 - margin, uhi = (float)(iu0 + kTU) + margin;

    auto centre_u = [&](int ix, int iy) -> float {
        const float xcf = ((float)ix + g.wx) * g.dx;
        const float ycf = ((float)iy + g.wy) * g.dy;
        const float tp = xcf * v.cos_a - ycf * v.sin_a;
        const float ds = g.sad + xcf * v.sin_a + ycf * v.cos_a;
        const float r = __fdividef(tp, ds);
        float u;
        if (g.det == 1) {
            u = g.sdd_du * r;
        } else if (g.det == 0) {
            u = g.sdd_du * atanf(r);
        } else {  // arc (candidate search only; the footprints are exact)
            const float gam = atanf(r);
            u = (gam + asinf(g.sad_add * sinf(gam))) * g.add / g.du;
        }
        return u - g.wu + 0.5f;
    };

    // 1. candidate interval of every line (binary search on the monotone centre projection)
    for (int L = t; L < nlines; L += NT) {
        auto f = [&](int p) { return rows ? centre_u(p, L) : centre_u(L, p); };
        const bool inc = f(npos - 1) >= f(0);
        int lo = 0, hi = npos;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float fm = f(mid);
            if (inc ? (fm < ulo) : (fm > uhi)) lo = mid + 1; else hi = mid;
        }
        const int first = lo;
        hi = npos;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float fm = f(mid);
            if (inc ? (fm > uhi) : (fm < ulo)) hi = mid; else lo = mid + 1;
        }
        line_start[L] = first;
        line_off[L] = lo - first;  // count, turned into offsets below
    }
    __syncthreads();
    // 2. exclusive scan of the counts
    {
        const int per = (nlines + NT - 1) / NT;
        const int b = t * per, e = min(b + per, nlines);
        int sum = 0;
        for (int L = b; L < e; L++) sum += line_off[L];
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += n;
        }
        if (lane == 31) s_warp_tot[warp] = incl;
        __syncthreads();
        int wbase = 0;
        for (int w = 0; w < warp; w++) wbase += s_warp_tot[w];
        int run = wbase + incl - sum;
        __syncthreads();
        for (int L = b; L < e; L++) {
            const int c = line_off[L];
            line_off[L] = run;
            run += c;
        }
        if (t == NT - 1) line_off[nlines] = run;
    }
    __syncthreads();
    const int ncand = line_off[nlines];
    const float fnz = (float)g.nz;
    const int nzm1 = g.nz - 1;
    const float fnzm1 = (float)nzm1;
    const int rows_per_pass = 4 * R;

    for (int c0 = 0; c0 < ncand; c0 += NT) {
        // 3. exact footprints of this chunk of candidates
        {
            const int c = c0 + t;
            bool valid = false;
            if (c < ncand) {
                int a = 0, bnd = nlines - 1;  // last line with line_off <= c
                while (a < bnd) {
                    const int mid = (a + bnd + 1) >> 1;
                    if (line_off[mid] <= c) a = mid; else bnd = mid - 1;
                }
                const int pos = line_start[a] + (c - line_off[a]);
                const int ix = rows ? pos : a, iy = rows ? a : pos;
                const int col = iy * g.nx + ix;
                if (map[col]) {
                    const ColumnFP fp = column_footprint<METHOD>(g, v, ix, iy);
                    if (fp.hit && fp.iumax >= iu0 && fp.iumin <= iu0 + kTU - 1) {
                        const int jlo = max(fp.iumin, iu0) - iu0, jhi = min(fp.iumax, iu0 + kTU - 1) - iu0;
                        const float scl = fp.ampu * fp.zinc;
#pragma unroll
                        for (int j = 0; j < kTU; j++) {
                            float w = 0.0f;
                            if (j >= jlo && j <= jhi)
                                w = u_weight<METHOD>(iu0 + j, fp.iumin, fp.iumax, fp.p0, fp.p1, fp.p2, fp.p3) * scl;
                            s_wf[t * kTU + j] = w;
                        }
                        const float b0 = fp.vstart + 0.5f;
                        const float btop = fmaf(fnz, fp.zinc, b0);
                        const int rlo = max((int)floorf(b0) - 1, 0);
                        const int rhi = min((int)floorf(btop) + 1, nv - 1);
                        if (rlo <= rhi) {
                            valid = true;
                            s_col[t] = col;
                            s_b0[t] = b0;
                            s_iz[t] = 1.0f / fp.zinc;
                            s_rlo[t] = rlo;
                            s_rhi[t] = rhi;
                            s_j[t] = jlo | (jhi << 8);
                        }
                    }
                }
            }
            if (!valid) s_j[t] = -1;
        }
        __syncthreads();
        // 4. row quads: R(iv) = X(iv+1) - X(iv) from the column's prefix pairs
        const int nslot = min(NT, ncand - c0);
        for (int s = grp; s < nslot; s += groups) {
            const int jj = s_j[s];
            if (jj < 0) continue;
            const int rlo = s_rlo[s], rhi = s_rhi[s];
            const float b0 = s_b0[s], izc = s_iz[s];
            const float *x = xs + (size_t)s_col[s] * (PAIRS ? 2 * (g.nz + 1) : g.xstride);
            const int jlo = jj & 0xff, jhi = jj >> 8;
            // groups of one warp own all their accumulator rows, so the warp walks the
            // candidate's own rows from rlo (128 per pass); wider groups own fixed bands
            const bool walk = R == 32;
            const int pstart = walk ? (rlo & ~3) : 0, pend = walk ? rhi + 1 : nv;
            for (int pbase = pstart; pbase < pend; pbase += rows_per_pass) {
                const int wrow = pbase + 128 * gwarp;  // first row of this warp's 128
                if (wrow > rhi || wrow + 127 < rlo) continue;  // warp-uniform
                const int iv0 = wrow + 4 * lane;
                const float f0 = small_int_to_float(iv0) - b0;
                float X0, X1, X2, X3;
                X0 = column_integral<PAIRS>(x, fminf(fmaxf(f0 * izc, 0.0f), fnz), nzm1, fnzm1);
                X1 = column_integral<PAIRS>(x, fminf(fmaxf((f0 + 1.0f) * izc, 0.0f), fnz), nzm1, fnzm1);
                X2 = column_integral<PAIRS>(x, fminf(fmaxf((f0 + 2.0f) * izc, 0.0f), fnz), nzm1, fnzm1);
                X3 = column_integral<PAIRS>(x, fminf(fmaxf((f0 + 3.0f) * izc, 0.0f), fnz), nzm1, fnzm1);
                float X4 = __shfl_down_sync(kFull, X0, 1);
                if (lane == 31) X4 = column_integral<PAIRS>(x, fminf(fmaxf((f0 + 4.0f) * izc, 0.0f), fnz), nzm1, fnzm1);
                if (iv0 <= rhi && iv0 + 3 >= rlo && iv0 < nv) {
                    const float R0 = X1 - X0, R1 = X2 - X1, R2 = X3 - X2, R3 = X4 - X3;
                    float4 *a = gacc + (iv0 >> 2);
                    for (int j = jlo; j <= jhi; j++) {
                        const float w = s_wf[s * kTU + j];
                        float4 r = a[j * nq];
                        r.x = fmaf(w, R0, r.x); r.y = fmaf(w, R1, r.y);
                        r.z = fmaf(w, R2, r.z); r.w = fmaf(w, R3, r.w);
                        a[j * nq] = r;
                    }
                }
            }
        }
        __syncthreads();
    }
    // 5. sum of the groups (in group order), axial amplitude and store
    const size_t obase = (size_t)k * g.nu * nv;
    const float *accf = reinterpret_cast<const float *>(acc4);
    const int gstride = kTU * 4 * nq;
    for (int j = 0; j < kTU; j++) {
        const int iu = iu0 + j;
        if (iu >= g.nu) break;
        for (int iv = t; iv < nv; iv += NT) {
            float a = accf[j * 4 * nq + iv];
#pragma unroll
            for (int q = 1; q < groups; q++) a += accf[q * gstride + j * 4 * nq + iv];
            store_from_float(proj, obase + (size_t)iu * nv + iv, a * ampv[(size_t)iu * nv + iv], out_dtype);
        }
    }
}

// Views per group of the forward projector's launch order.
constexpr int kViewGroup = 32;

// Detector-column group bx and launch view by of the forward projector's linear block
// L: the launch views in groups of kViewGroup consecutive ones (the last group may be
// shorter), and within a group the blocks of one detector-column group over all its
// views, then the next column group -- neighbouring views share candidate columns in L2.
__device__ __forceinline__ void view_grouped_block(int L, int ngx, int vc, int &bx, int &by) {
    const int per = ngx * kViewGroup;
    const int G = L / per, r = L - G * per;
    const int n = min(kViewGroup, vc - G * kViewGroup);  // views of this group
    bx = r / n;
    by = G * kViewGroup + (r - bx * n);
}

template <int METHOD, int GROUPS, bool PAIRS>
__global__ void __launch_bounds__(kProjMaxThreads) proj_kernel(Geom g, const View *__restrict__ views,
                                                               const float *__restrict__ xs,
                                                               const float *__restrict__ ampv,
                                                               const uint8_t *__restrict__ map,
                                                               void *__restrict__ proj, int out_dtype,
                                                               int view_begin, int view_stride, float margin,
                                                               int ngx, int vc) {
    extern __shared__ float4 acc4_smem[];
    int bx, by;
    view_grouped_block(blockIdx.x, ngx, vc, bx, by);
    proj_block<METHOD, GROUPS, PAIRS>(g, views, xs, ampv, map, proj, out_dtype, view_begin, view_stride, margin,
                                      acc4_smem, bx, by);
}

// ---------------------------------------------------------------------------
// A with the candidates' prefix columns staged in shared memory by bulk copies.
//
// Same decomposition and arithmetic as proj_block: one block per (group of kTU
// detector columns, view), candidate columns from the monotone projected centres of
// the volume lines, exact footprints per candidate, rows accumulated as
// w_u * ampu * zinc * (X(iv+1) - X(iv)) by the thread that owns them.  What changes is
// where X comes from: the valid candidates of a chunk are packed into a list, and
// their whole prefix columns (g.xstride floats, X[nz] repeated at the top) are copied
// from global memory into shared memory by the copy engine (cp.async.bulk, completion
// counted in bytes on an mbarrier), `slots` columns at a time into one of two buffers,
// so that the copies of the next slots overlap the row loop over the current ones.  The
// row loop then reads X from shared memory (32-bit addresses, no global gathers).
// ---------------------------------------------------------------------------
constexpr int kMbarPolls = 1 << 22;  // bound of every mbarrier wait (a copy normally lands in microseconds)

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// Makes the initialised barriers visible to the copy engine (async proxy).
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// One arrival that also announces `bytes` of copies to complete on this phase.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// One plain arrival (release: the arriving thread's earlier shared-memory reads are done).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16), its
// bytes counted on `bar`.  No multicast: the destination is this block's own memory.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// Waits for the phase of the given parity to complete; false after kMbarPolls polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    const uint32_t a = smem_addr(bar);
    for (int i = 0; i < kMbarPolls; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// X(s) of a staged column, s clamped to [0, nz] (X[nz + 1] = X[nz] is part of the copy).
// xadj: the column's shared-memory address minus 4 * 0x4B000000 (mod 2^32), so that the
// address of X[floor(s)] is xadj + 4 * bits(s + 2^23 rounded down).
__device__ __forceinline__ float staged_integral(uint32_t xadj, float s, float fnz) {
    s = fminf(fmaxf(s, 0.0f), fnz);
    const float t = __fadd_rd(s, kTwo23);
    const uint32_t a = xadj + (__float_as_uint(t) << 2);
    float x0, x1;
    asm volatile("ld.shared.f32 %0, [%2];\n\tld.shared.f32 %1, [%2+4];" : "=f"(x0), "=f"(x1) : "r"(a));
    return fmaf(s - (t - kTwo23), x1 - x0, x0);
}
__device__ __forceinline__ float lds_f32(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ float4 lds_f32x4(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
// acc += w * (r0, r1, r2, r3) on the float4 at shared address a.
__device__ __forceinline__ void acc_add4(uint32_t a, float w, float r0, float r1, float r2, float r3) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    v.x = fmaf(w, r0, v.x); v.y = fmaf(w, r1, v.y); v.z = fmaf(w, r2, v.z); v.w = fmaf(w, r3, v.w);
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}

// Dynamic shared-memory layout of the staged forward projector: four mbarriers (first, so
// that a persistent block keeps them across work items of different shapes), the
// accumulators, the two stage buffers, the packed candidate table, the
// line tables.
struct StagedSmem {
    int nq, nt, nlines, groups, slots, xstride;
    __host__ __device__ size_t acc_bytes() const { return (size_t)groups * kTU * nq * 16; }
    __host__ __device__ size_t stage_floats() const { return (size_t)slots * xstride; }  // one buffer
    __host__ __device__ size_t bytes() const {
        return 32 + acc_bytes() + 2 * stage_floats() * 4 + (size_t)nt * (5 + kTU) * 4 +
               (size_t)(2 * nlines + 1 + 32) * 4;
    }
};

// Error flag bit of a stage wait that ran out (ctsim_plan_check reports the flag).
constexpr int kErrStageWait = 4;

// The stage buffers form a two-deep full/empty pipeline: bar[b] ("full", one arrival plus
// the copies' bytes) completes when buffer b holds its slots, bar[2 + b] ("empty", one
// arrival per warp) when every warp has finished reading it.  A thread's `phase` holds the
// parity of the next completion it waits for: bit b for full[b], bit 2 + b for empty[b].
// The empty bits start at 1, the parity of the phase before a fresh barrier's first,
// which counts as complete, so the first copies into each buffer do not wait.
constexpr unsigned kStagedPhase0 = 0xCu;

__device__ __forceinline__ void staged_bars_init(uint64_t *bar) {
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init(&bar[2], blockDim.x >> 5);
        mbar_init(&bar[3], blockDim.x >> 5);
        mbar_init_fence();
    }
    __syncthreads();
}

// Candidate intervals of the lines for detector columns [iu0, iu0 + kTU) of view v:
// line_start[L], and line_off[L] the exclusive scan of the counts (line_off[nlines] =
// the total).  All threads of the block call it; ends with a block barrier.
__device__ __forceinline__ int candidate_lines(const Geom &g, const View &v, int iu0, float margin, bool rows,
                                               int *line_start, int *line_off, int *s_warp_tot) {
    const int NT = blockDim.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nlines = rows ? g.ny : g.nx;
    const int npos = rows ? g.nx : g.ny;
    const float ulo = (float)iu0 - margin, uhi = (float)(iu0 + kTU) + margin;
    auto centre_u = [&](int ix, int iy) -> float {
        const float xcf = ((float)ix + g.wx) * g.dx;
        const float ycf = ((float)iy + g.wy) * g.dy;
        const float tp = xcf * v.cos_a - ycf * v.sin_a;
        const float ds = g.sad + xcf * v.sin_a + ycf * v.cos_a;
        const float r = __fdividef(tp, ds);
        float u;
        if (g.det == 1) {
            u = g.sdd_du * r;
        } else if (g.det == 0) {
            u = g.sdd_du * atanf(r);
        } else {  // arc (candidate search only; the footprints are exact)
            const float gam = atanf(r);
            u = (gam + asinf(g.sad_add * sinf(gam))) * g.add / g.du;
        }
        return u - g.wu + 0.5f;
    };
    for (int L = t; L < nlines; L += NT) {
        auto f = [&](int p) { return rows ? centre_u(p, L) : centre_u(L, p); };
        const bool inc = f(npos - 1) >= f(0);
        int lo = 0, hi = npos;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float fm = f(mid);
            if (inc ? (fm < ulo) : (fm > uhi)) lo = mid + 1; else hi = mid;
        }
        const int first = lo;
        hi = npos;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float fm = f(mid);
            if (inc ? (fm > uhi) : (fm < ulo)) hi = mid; else lo = mid + 1;
        }
        line_start[L] = first;
        line_off[L] = lo - first;
    }
    __syncthreads();
    const int per = (nlines + NT - 1) / NT;
    const int b = t * per, e = min(b + per, nlines);
    int sum = 0;
    for (int L = b; L < e; L++) sum += line_off[L];
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += n;
    }
    if (lane == 31) s_warp_tot[warp] = incl;
    __syncthreads();
    int wbase = 0;
    for (int w = 0; w < warp; w++) wbase += s_warp_tot[w];
    int run = wbase + incl - sum;
    __syncthreads();
    for (int L = b; L < e; L++) {
        const int c = line_off[L];
        line_off[L] = run;
        run += c;
    }
    if (t == NT - 1) line_off[nlines] = run;
    __syncthreads();
    return line_off[nlines];
}

// The work of one block.  bar: the block's four stage mbarriers (initialised once per
// block by staged_bars_init); phase: their next-completion parities, carried across the
// items of a persistent block (kStagedPhase0 at the start); acc4: the shared memory past
// the mbarriers.  Returns false when a stage wait ran out (the block has then set
// kErrStageWait, waited for its copies in flight and must stop).
template <int METHOD, int GROUPS>
__device__ __forceinline__ bool proj_staged_block(const Geom g, const View *__restrict__ views,
                                                  const float *__restrict__ xs, const float *__restrict__ ampv,
                                                  const uint8_t *__restrict__ map, void *__restrict__ proj,
                                                  int out_dtype, int view_begin, int view_stride, float margin,
                                                  int slots, int *__restrict__ err, float4 *acc4, uint64_t *bar,
                                                  unsigned &phase, int bx, int by) {
    const int NT = blockDim.x;
    const int R = NT / GROUPS;
    const int nv = g.nv;
    const int nq = (nv + 3) >> 2;
    const int nlines0 = max(g.nx, g.ny);
    const int xst = g.xstride;
    StagedSmem L{nq, NT, nlines0, GROUPS, slots, xst};
    float *stage = reinterpret_cast<float *>(acc4 + GROUPS * kTU * nq);  // [2][slots][xst]
    // per candidate slot: {-b0 / zinc, 1 / zinc, rlo | rhi << 16, jlo | jhi << 8} (one 16-byte load)
    // (all three indexed by the candidate's position among the chunk's valid candidates)
    float4 *c_prm = reinterpret_cast<float4 *>(stage + 2 * L.stage_floats());
    int *c_col = reinterpret_cast<int *>(c_prm + NT);
    float *c_w = reinterpret_cast<float *>(c_col + NT);  // [NT][kTU]
    int *line_start = reinterpret_cast<int *>(c_w + NT * kTU);
    int *line_off = line_start + nlines0;
    int *s_warp_tot = line_off + nlines0 + 1;  // [32]

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int grp = GROUPS == 1 ? 0 : t / R;
    const int gwarp = GROUPS == 1 ? warp : (t - grp * R) >> 5;
    const int iu0 = bx * kTU;
    const View v = views[view_begin + by * view_stride];
    for (int i = t; i < GROUPS * kTU * nq; i += NT) acc4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 *gacc = acc4 + grp * kTU * nq;
    // 32-bit shared addresses of the row loop's tables
    const uint32_t acc_u32 = smem_addr(gacc), nq16 = 16u * (uint32_t)nq;
    const uint32_t prm_u32 = smem_addr(c_prm), w_u32 = smem_addr(c_w);
    const float fnz = (float)g.nz;
    // rows iv0 .. iv0 + 3 (f0 = iv0 as float) of one candidate: X at the five row edges from
    // the staged column (xadj), R = X(iv + 1) - X(iv), added with the weights at wq (16-byte
    // aligned, the first for the candidate's first column) into the accumulator columns at aq
    // (pjn + 1 of them).  Boundary iv sits at s = iv / zinc -
    // b0 / zinc (psa, piz), one rounding from iv alone, so a row's value does not depend on
    // which lane, warp or pass evaluates it; rows outside the column's shadow have both
    // edges clamped to the same end of the column and add exactly 0 (no per-lane test).
    auto staged_rows = [&](int iv0, float f0, float psa, float piz, uint32_t xadj, uint32_t wq, uint32_t aq,
                           int pjn) {
        const float X0 = staged_integral(xadj, fmaf(f0, piz, psa), fnz);
        const float X1 = staged_integral(xadj, fmaf(f0 + 1.0f, piz, psa), fnz);
        const float X2 = staged_integral(xadj, fmaf(f0 + 2.0f, piz, psa), fnz);
        const float X3 = staged_integral(xadj, fmaf(f0 + 3.0f, piz, psa), fnz);
        const float X4 = staged_integral(xadj, fmaf(f0 + 4.0f, piz, psa), fnz);
        if (iv0 < nv) {
            const float R0 = X1 - X0, R1 = X2 - X1, R2 = X3 - X2, R3 = X4 - X3;
            const uint32_t a = aq + 4u * (uint32_t)iv0;  // float4 of rows iv0 .. iv0 + 3
            const float4 w4 = lds_f32x4(wq);  // the candidate's first four weights
            acc_add4(a, w4.x, R0, R1, R2, R3);
            if (pjn > 0) {
                acc_add4(a + nq16, w4.y, R0, R1, R2, R3);
                if (pjn > 1) {
                    acc_add4(a + 2u * nq16, w4.z, R0, R1, R2, R3);
                    if (pjn > 2) {
                        acc_add4(a + 3u * nq16, w4.w, R0, R1, R2, R3);
                        for (int j = 4; j <= pjn; j++)
                            acc_add4(a + (uint32_t)j * nq16, lds_f32(wq + 4u * j), R0, R1, R2, R3);
                    }
                }
            }
        }
    };
    const bool rows = fabsf(v.cos_a) >= fabsf(v.sin_a);
    const int nlines = rows ? g.ny : g.nx;
    const int ncand = candidate_lines(g, v, iu0, margin, rows, line_start, line_off, s_warp_tot);
    const int rows_per_pass = 4 * R;
    const unsigned col_bytes = (unsigned)xst * 4u;
    int buf0 = 0;   // buffer of the next chunk's first slots
    int vbase = 0;  // valid candidates of the earlier chunks

    for (int c0 = 0; c0 < ncand; c0 += NT) {
        // 1. exact footprint of candidate c0 + t; the valid candidates' scalars, weights and
        // columns are packed in candidate order
        bool valid = false;
        int my_col = 0;
        float4 my_prm;
        float my_w[kTU];
        {
            const int c = c0 + t;
            if (c < ncand) {
                int a = 0, bnd = nlines - 1;  // last line with line_off <= c
                while (a < bnd) {
                    const int mid = (a + bnd + 1) >> 1;
                    if (line_off[mid] <= c) a = mid; else bnd = mid - 1;
                }
                const int pos = line_start[a] + (c - line_off[a]);
                const int ix = rows ? pos : a, iy = rows ? a : pos;
                const int col = iy * g.nx + ix;
                if (map[col]) {
                    const ColumnFP fp = column_footprint<METHOD>(g, v, ix, iy);
                    if (fp.hit && fp.iumax >= iu0 && fp.iumin <= iu0 + kTU - 1) {
                        const int jlo = max(fp.iumin, iu0) - iu0, jhi = min(fp.iumax, iu0 + kTU - 1) - iu0;
                        const float scl = fp.ampu * fp.zinc;
                        // weight i for detector column iu0 + jlo + i (16-byte loads in the row loop)
#pragma unroll
                        for (int i = 0; i < kTU; i++) {
                            float w = 0.0f;
                            if (jlo + i <= jhi)
                                w = u_weight<METHOD>(iu0 + jlo + i, fp.iumin, fp.iumax, fp.p0, fp.p1, fp.p2, fp.p3) *
                                    scl;
                            my_w[i] = w;
                        }
                        const float b0 = fp.vstart + 0.5f;
                        const float btop = fmaf(fnz, fp.zinc, b0);
                        const int rlo = max((int)floorf(b0) - 1, 0);
                        const int rhi = min((int)floorf(btop) + 1, nv - 1);
                        if (rlo <= rhi) {
                            valid = true;
                            const float izc = 1.0f / fp.zinc;
                            my_col = col;
                            // s(iv) = iv / zinc - b0 / zinc
                            my_prm = make_float4(-b0 * izc, izc, __int_as_float(rlo | (rhi << 16)),
                                                 __int_as_float(jlo | (jhi << 8)));
                        }
                    }
                }
            }
        }
        const unsigned bal = __ballot_sync(kFull, valid);
        if (lane == 0) s_warp_tot[warp] = __popc(bal);
        __syncthreads();
        int base = 0, nval = 0;
        for (int w = 0; w < (NT >> 5); w++) {
            const int n = s_warp_tot[w];
            base += w < warp ? n : 0;
            nval += n;
        }
        if (valid) {
            const int q = base + __popc(bal & ((1u << lane) - 1u));
            c_col[q] = my_col;
            c_prm[q] = my_prm;
#pragma unroll
            for (int j = 0; j < kTU; j++) c_w[q * kTU + j] = my_w[j];
        }
        __syncthreads();

        // 2. the packed candidates, `slots` at a time: warp 0 issues the copies of the next
        // slots into the other buffer once every warp has released it, while the warps run
        // the rows of the current ones; each warp releases a buffer when it is done with it
        const int nsub = (nval + slots - 1) / slots;
        bool failed = false;
        auto issue = [&](int sub, int buf) {
            const int p0 = sub * slots, n = min(slots, nval - p0);
            const bool free = mbar_wait(&bar[2 + buf], (phase >> (2 + buf)) & 1u);
            phase ^= 4u << buf;
            failed |= !free;
            // a buffer that was not released gets no copies: its full phase completes empty
            // and the block stops at the end of the chunk
            if (lane == 0) mbar_arrive_expect(&bar[buf], free ? (unsigned)n * col_bytes : 0u);
            __syncwarp();
            if (!free) return;
            float *dst = stage + (size_t)buf * L.stage_floats();
            for (int i = lane; i < n; i += 32)
                bulk_copy_g2s(dst + (size_t)i * xst, xs + (size_t)c_col[p0 + i] * xst, col_bytes, &bar[buf]);
        };
        if (nsub > 0 && warp == 0) issue(0, buf0);
        for (int sub = 0; sub < nsub; sub++) {
            const int buf = (buf0 + sub) & 1;
            if (sub + 1 < nsub && warp == 0) issue(sub + 1, buf ^ 1);
            failed |= !mbar_wait(&bar[buf], (phase >> buf) & 1u);
            phase ^= 1u << buf;
            const uint32_t sb = smem_addr(stage + (size_t)buf * L.stage_floats()) - (0x4B000000u << 2);
            const int p0 = sub * slots, p1 = min(nval, p0 + slots);
            // group g takes the valid candidates whose position in the block's whole sequence of
            // valid candidates (vbase + p) is g mod GROUPS, in order: the same split and order
            // whatever the chunk, row-thread or slot counts
            const int pstart0 = p0 + (((grp - vbase - p0) % GROUPS) + GROUPS) % GROUPS;
            if (R == 32) {
                // one-warp groups walk each candidate's own rows (every row of the group is theirs)
                for (int p = pstart0; p < p1; p += GROUPS) {
                    const float4 prm = lds_f32x4(prm_u32 + 16u * (uint32_t)p);
                    const int rr = __float_as_int(prm.z), jj = __float_as_int(prm.w);
                    const int prlo = rr & 0xffff, prhi = rr >> 16;
                    const int pjlo = jj & 0xff;
                    const uint32_t xadj = sb + (uint32_t)((p - p0) * xst) * 4u;
                    for (int wrow = prlo & ~3; wrow <= prhi; wrow += 128)
                        staged_rows(wrow + 4 * lane, small_int_to_float(wrow + 4 * lane), prm.x, prm.y, xadj,
                                    w_u32 + 4u * (uint32_t)(p * kTU), acc_u32 + nq16 * (uint32_t)pjlo,
                                    (jj >> 8) - pjlo);
                }
            } else {
                // fixed bands: warp gwarp owns rows pbase + 128 gwarp .. + 127 of each pass
                for (int pbase = 0; pbase < nv; pbase += rows_per_pass) {
                    const int wrow = pbase + 128 * gwarp;
                    const int iv0 = wrow + 4 * lane;
                    const float f0 = small_int_to_float(iv0);
                    for (int p = pstart0; p < p1; p += GROUPS) {
                        const float4 prm = lds_f32x4(prm_u32 + 16u * (uint32_t)p);
                        const int rr = __float_as_int(prm.z), jj = __float_as_int(prm.w);
                        if (wrow > (rr >> 16) || wrow + 127 < (rr & 0xffff)) continue;  // warp-uniform
                        const int pjlo = jj & 0xff;
                        staged_rows(iv0, f0, prm.x, prm.y, sb + (uint32_t)((p - p0) * xst) * 4u,
                                    w_u32 + 4u * (uint32_t)(p * kTU), acc_u32 + nq16 * (uint32_t)pjlo,
                                    (jj >> 8) - pjlo);
                    }
                }
            }
            // this warp is done with buffer `buf`
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar[2 + buf]);
        }
        // every warp is done with this chunk's candidate tables before the next chunk
        // rewrites them
        if (__syncthreads_or(failed)) {
            if (t == 0) atomicOr(err, kErrStageWait);
            // let copies still in flight land before the block stops (bounded waits: a
            // phase that completed, or never began, returns at once)
            mbar_wait(&bar[0], (phase & 1u) ^ 1u);
            mbar_wait(&bar[1], ((phase >> 1) & 1u) ^ 1u);
            return false;
        }
        buf0 = (buf0 + nsub) & 1;
        vbase += nval;
    }
    if (ncand == 0) __syncthreads();
    // 3. sum of the groups (in group order), axial amplitude and store
    const size_t obase = (size_t)by * g.nu * nv;
    const float *accf = reinterpret_cast<const float *>(acc4);
    const int gstride = kTU * 4 * nq;
    for (int j = 0; j < kTU; j++) {
        const int iu = iu0 + j;
        if (iu >= g.nu) break;
        for (int iv = t; iv < nv; iv += NT) {
            float a = accf[j * 4 * nq + iv];
#pragma unroll
            for (int q = 1; q < GROUPS; q++) a += accf[q * gstride + j * 4 * nq + iv];
            store_from_float(proj, obase + (size_t)iu * nv + iv, a * ampv[(size_t)iu * nv + iv], out_dtype);
        }
    }
    return true;
}

template <int METHOD, int GROUPS>
__global__ void __launch_bounds__(kProjMaxThreads, 3) proj_staged_kernel(Geom g, const View *__restrict__ views,
                                                                      const float *__restrict__ xs,
                                                                      const float *__restrict__ ampv,
                                                                      const uint8_t *__restrict__ map,
                                                                      void *__restrict__ proj, int out_dtype,
                                                                      int view_begin, int view_stride, float margin,
                                                                      int slots, int *__restrict__ err, int ngx,
                                                                      int vc) {
    extern __shared__ float4 smem_staged[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_staged);
    staged_bars_init(bar);
    unsigned phase = kStagedPhase0;
    int bx, by;
    view_grouped_block(blockIdx.x, ngx, vc, bx, by);
    proj_staged_block<METHOD, GROUPS>(g, views, xs, ampv, map, proj, out_dtype, view_begin, view_stride, margin,
                                      slots, err, smem_staged + 2, bar, phase, bx, by);
}

// ---------------------------------------------------------------------------
// FDK voxel-driven bilinear backprojection (geom/cbct/cbct_back.c:7-133): warp
// per column, lanes along z.  Per-view column quantities (u, w2, w2s) are computed
// by lane j for view k0+j and broadcast; every voxel accumulates the views in the
// reference's order with its exact float operations.
// ---------------------------------------------------------------------------
// SUM: the FP32 image holds the view sum of earlier view chunks (scale 1), which the
// kernel continues in the same view order (separate instantiations).
// One sinogram sample of storage type DT (kF32, kBF16, kF16) as float (exact widening).
template <int DT>
__device__ __forceinline__ float ld_sino(const void *__restrict__ base, size_t i) {
    if (DT == kBF16) return __uint_as_float((unsigned)__ldg(static_cast<const unsigned short *>(base) + i) << 16);
    if (DT == kF16) return __half2float(__ushort_as_half(__ldg(static_cast<const unsigned short *>(base) + i)));
    return __ldg(static_cast<const float *>(base) + i);
}

// DT: the sinogram's storage type, read as it is (widening to FP32 is exact, so the
// result equals that of an FP32 copy bit for bit).
template <int MODE, int MZ, bool SUM = false, int DT = kF32>
__global__ void __launch_bounds__(256) pd_kernel(Geom g, const View *__restrict__ views,
                                                 const void *__restrict__ proj, const uint8_t *__restrict__ map,
                                                 void *__restrict__ image, int out_dtype, int view_begin,
                                                 int view_stride, int view_count, float scale) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (g.nx + 7) >> 3;
    const int iy = blockIdx.x / tiles_x;
    const int ix = (blockIdx.x % tiles_x) * 8 + warp;
    if (ix >= g.nx || iy >= g.ny) return;
    // per view of the current 32-view chunk, written by the view's own lane:
    // {wul, omu, w2, w2s}, {couch, 1 if u is on the detector else 0, bits of the detector
    // column's element offset}
    __shared__ float4 vtab[8][32][2];
    const size_t nxy = (size_t)g.nx * g.ny;
    const size_t nuv = (size_t)g.nu * g.nv;
    const bool on = map[iy * g.nx + ix] != 0;
    const float xc = fmul(fadd((float)ix, g.wx), g.dx);
    const float yc = fmul(fadd((float)iy, g.wy), g.dy);
    const int zpass = 32 * MZ;
    for (int iz0 = 0; iz0 < g.nz; iz0 += zpass) {
        const int izn = min(zpass, g.nz - iz0);
        float acc[MZ], zc0[MZ];
#pragma unroll
        for (int m = 0; m < MZ; m++) {
            acc[m] = 0.0f;
            zc0[m] = fmul(fadd((float)(iz0 + lane + 32 * m), g.wz_pd), g.dz);  // (iz + wz) * dz, cbct_back.c:100
        }
        if (SUM) {
            const float *src = static_cast<const float *>(image) + (size_t)(iz0 + lane) * nxy + (size_t)iy * g.nx + ix;
#pragma unroll
            for (int m = 0; m < MZ; m++)
                if (lane + 32 * m < izn) acc[m] = src[(size_t)(32 * m) * nxy];
        }
        if (on) {
            for (int k0 = 0; k0 < view_count; k0 += 32) {
                constexpr bool OFF = MODE != kPdClamp, VAR = MODE == kPdVar;
                float u = -1.0f, w2 = 0.0f, w2s = 0.0f, couch = 0.0f;
                const int kl = k0 + lane;
                if (kl < view_count) {
                    const View v = views[view_begin + kl * view_stride];
                    const float xr = fsub(fmul(xc, v.cos_a), fmul(yc, v.sin_a));
                    const float yr = fadd(fmul(xc, v.sin_a), fmul(yc, v.cos_a));
                    const float den = fadd(g.sad, yr);
                    if (g.det == 1) {  // cbct_back.c:68-77
                        w2 = fdiv(g.sdd, den);
                        w2s = fmul(w2, w2);
                        u = fsub(fdiv(fmul(xr, w2), g.du), g.wu);
                    } else {           // cbct_back.c:78-88, cbct_back_var.c:68-77
                        const float xo = fsub(xr, VAR ? g.roff_var : g.roff);
                        const double at = atan((double)fdiv(xo, den));
                        u = (float)__dsub_rn(__ddiv_rn(__dmul_rn(at, (double)g.sdd), (double)g.du), (double)g.wu);
                        w2s = fdiv(fmul(g.sdd, g.sdd), fadd(fmul(den, den), fmul(xo, xo)));
                        w2 = fdiv(g.sdd, den);
                    }
                    couch = VAR ? v.wz : v.couch_pd;  // back,var: the couch shift is in wz
                }
                {
                    // this lane's view: the detector column and u weights (cbct_back.c:90-99)
                    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = make_float4(couch, __int_as_float(0), 0.f, 0.f);
                    if (kl < view_count && u >= g.u_lo && u <= g.u_hi) {  // cbct_back.c:90
                        float fiu;
                        const int iu = floor_pos(u, &fiu);
                        const float wul = fsub(u, fiu);
                        a = make_float4(wul, fsub(1.0f, wul), w2, w2s);
                        const unsigned long long pv = (unsigned long long)kl * nuv + (unsigned long long)iu * g.nv;
                        b.y = __int_as_float(1);
                        b.z = __uint_as_float((unsigned)pv);
                        b.w = __uint_as_float((unsigned)(pv >> 32));
                    }
                    __syncwarp();  // the previous chunk's reads are done
                    vtab[warp][lane][0] = a;
                    vtab[warp][lane][1] = b;
                }
                __syncwarp();
                const int nk = min(32, view_count - k0);
                for (int j = 0; j < nk; j++) {
                    const float4 b = vtab[warp][j][1];
                    if (__float_as_int(b.y) == 0) continue;  // u off the detector
                    const float4 a = vtab[warp][j][0];
                    const float wul = a.x, omu = a.y, w2j = a.z, w2sj = a.w, cj = b.x;
                    const size_t pv = ((size_t)__float_as_uint(b.w) << 32) | __float_as_uint(b.z);  // element offset
#pragma unroll
                    for (int m = 0; m < MZ; m++) {
                        if (lane + 32 * m < izn) {
                            // (iz + wz) * dz + couch (cbct_back.c:100); back,var: (iz + wz) * dz with
                            // the view's wz (cbct_back_var.c:41, :89)
                            const float zc = VAR ? fmul(fadd((float)(iz0 + lane + 32 * m), cj), g.dz)
                                                 : fadd(zc0[m], cj);
                            float vv = fsub(div_by(fmul(zc, w2j), g.dv, g.rdv), g.wv);  // cbct_back.c:102
                            bool use = true;
                            if (OFF) {
                                use = vv >= g.v_lo && vv <= g.v_hi;  // cbct_back.c:105-108
                            } else {
                                vv = vv > 0.5f ? vv : 0.5f;          // cbct_back.c:110-111
                                vv = vv < g.v_clamp_hi ? vv : g.v_clamp_hi;
                            }
                            if (use) {
                                float fiv;
                                const int iv = min(floor_pos(vv, &fiv), g.nv - 2);
                                const float wvl = fsub(vv, fiv);
                                const float omv = fsub(1.0f, wvl);
                                const size_t p = pv + iv;
                                const float s0 = fadd(fmul(omv, ld_sino<DT>(proj, p)), fmul(wvl, ld_sino<DT>(proj, p + 1)));
                                const float s1 = fadd(fmul(omv, ld_sino<DT>(proj, p + g.nv)),
                                                      fmul(wvl, ld_sino<DT>(proj, p + g.nv + 1)));
                                const float val = fadd(fmul(omu, s0), fmul(wul, s1));
                                // w2s * (...) (cbct_back.c:120); w2s * w2s * (...) (cbct_back_var.c:116)
                                acc[m] = fadd(acc[m], fmul(VAR ? fmul(w2sj, w2sj) : w2sj, val));
                            }
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int m = 0; m < MZ; m++) {
            const int dz = lane + 32 * m;
            if (dz < izn) {
                float r = on ? acc[m] : 0.0f;
                if (scale != 1.0f) r = r * scale;
                store_from_float(image, (size_t)(iz0 + dz) * nxy + (size_t)iy * g.nx + ix, r, out_dtype);
            }
        }
    }
}

__global__ void scale_kernel(float *__restrict__ y, size_t n, float s) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] *= s;
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
// The dynamic shared-memory limit is a per-function, per-device attribute shared by
// every plan, stream and captured graph of the process; it is only ever raised, so
// a launch recorded earlier (another request's stream, a CUDA graph) stays valid.
cudaError_t allow_dynamic_smem(const void *kfn, size_t bytes) {
    static std::mutex m;
    static std::map<std::pair<int, const void *>, size_t> granted;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(m);
    size_t &g = granted[{dev, kfn}];
    if (bytes <= g) return cudaSuccess;
    e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) g = bytes;
    return e;
}

// per warp: the u weights of 32 views and the row buffer; 4 spare floats past the last
// warp's buffer for the branch-free row reads
size_t back_smem_bytes(int qcap) { return ((size_t)8 * (32 * 17 + 32 * 8 + qcap) + 4) * sizeof(float); }

template <int METHOD, int MZ, bool VEC, int SRC, bool SUM>
static cudaError_t launch_back_mz(const Geom &g, const View *views, const void *ps, const float *ampv,
                                  const uint8_t *map, void *image, int out_dtype, int vb, int vs, int vc, float scale,
                                  int qcap, int *err, int y_begin, int y_end, cudaStream_t st) {
    const int tiles_x = (g.nx + 7) / 8;
    const int blocks = (y_end - y_begin) * tiles_x;
    if (blocks <= 0) return cudaSuccess;
    const size_t sm = back_smem_bytes(qcap);
    auto kfn = back_kernel<METHOD, MZ, VEC, SRC, SUM>;
    cudaError_t e = allow_dynamic_smem((const void *)kfn, sm);
    if (e != cudaSuccess) return e;
    kfn<<<blocks, 256, sm, st>>>(g, views, ps, map, image, out_dtype, vb, vs, vc, scale, qcap, err, ampv,
                                 y_begin * tiles_x);
    return cudaGetLastError();
}

cudaError_t launch_prescale(const void *proj, int in_dtype, const float *ampv, float *ps, size_t nuv, size_t n,
                            cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 32);
    prescale_kernel<<<blocks, 256, 0, st>>>(proj, in_dtype, ampv, ps, nuv, n);
    return cudaGetLastError();
}

cudaError_t launch_back(int method, int mz, const Geom &g, const View *views, const void *ps, const uint8_t *map,
                        void *image, int out_dtype, int vb, int vs, int vc, float scale, int qcap, int *err,
                        cudaStream_t st, bool accumulate, int y_begin, int y_end, int src, const float *ampv) {
    if (accumulate && (out_dtype != kF32 || scale != 1.0f || src != kSrcScaled)) return cudaErrorInvalidValue;
    if (src != kSrcScaled && src != kSrcBF16 && src != kSrcF16) return cudaErrorInvalidValue;
    if (src != kSrcScaled && !ampv) return cudaErrorInvalidValue;
    if (y_end < 0) y_end = g.ny;
    if (y_begin < 0 || y_end > g.ny || y_begin > y_end) return cudaErrorInvalidValue;
    const size_t align = src == kSrcScaled ? 16 : 8;  // one float4, or four 16-bit values, per load
    const bool vec = (g.nv % 4) == 0 && (reinterpret_cast<uintptr_t>(ps) % align) == 0 &&
                     (reinterpret_cast<uintptr_t>(ampv) % 16) == 0;
    // accumulate: the image holds the FP32 view sum of earlier views, which the kernel
    // continues (separate instantiations, so the plain kernel keeps its registers)
#define CTSIM_BACK_ARGS g, views, ps, ampv, map, image, out_dtype, vb, vs, vc, scale, qcap, err, y_begin, y_end, st
#define CTSIM_BACK_CASE(M, Z)                                                                            \
    if (method == M && mz == Z) {                                                                        \
        if (accumulate)                                                                                  \
            return vec ? launch_back_mz<M, Z, true, kSrcScaled, true>(CTSIM_BACK_ARGS)                   \
                       : launch_back_mz<M, Z, false, kSrcScaled, true>(CTSIM_BACK_ARGS);                 \
        if (src == kSrcBF16)                                                                             \
            return vec ? launch_back_mz<M, Z, true, kSrcBF16, false>(CTSIM_BACK_ARGS)                    \
                       : launch_back_mz<M, Z, false, kSrcBF16, false>(CTSIM_BACK_ARGS);                  \
        if (src == kSrcF16)                                                                              \
            return vec ? launch_back_mz<M, Z, true, kSrcF16, false>(CTSIM_BACK_ARGS)                     \
                       : launch_back_mz<M, Z, false, kSrcF16, false>(CTSIM_BACK_ARGS);                   \
        return vec ? launch_back_mz<M, Z, true, kSrcScaled, false>(CTSIM_BACK_ARGS)                      \
                   : launch_back_mz<M, Z, false, kSrcScaled, false>(CTSIM_BACK_ARGS);                    \
    }
    CTSIM_BACK_CASE(kDD, 1) CTSIM_BACK_CASE(kDD, 2) CTSIM_BACK_CASE(kDD, 4) CTSIM_BACK_CASE(kDD, 8)
    CTSIM_BACK_CASE(kTF, 1) CTSIM_BACK_CASE(kTF, 2) CTSIM_BACK_CASE(kTF, 4) CTSIM_BACK_CASE(kTF, 8)
#undef CTSIM_BACK_CASE
#undef CTSIM_BACK_ARGS
    return cudaErrorInvalidValue;
}

cudaError_t launch_prefix(const void *image, int in_dtype, float *xs, int nxy, int nz, bool pairs, int xstride,
                          cudaStream_t st) {
    const int blocks = (nxy + 31) / 32;
    if (pairs) prefix_kernel<true><<<blocks, 256, 0, st>>>(image, in_dtype, xs, nxy, nz, 0);
    else prefix_kernel<false><<<blocks, 256, 0, st>>>(image, in_dtype, xs, nxy, nz, xstride);
    return cudaGetLastError();
}

// Row threads R (one per 4 detector rows, whole warps, at most kProjMaxThreads) and
// candidate groups (1, 2, 4 or 8, with R * groups <= kProjMaxThreads).  Default: two
// groups wherever they fit (R <= 128, up to 512 rows) -- the fastest count on every
// shape measured on B200 (nv 72..384); one group above.  A plan's autotuner may pick
// another valid count.
static int proj_row_threads(int nv) {
    return std::min(kProjMaxThreads, std::max(32, ((nv + 3) / 4 + 31) / 32 * 32));
}
int proj_default_groups(int nv) { return proj_row_threads(nv) <= kProjMaxThreads / 2 ? 2 : 1; }
int proj_default_rows(int nv) { return proj_row_threads(nv); }
// rows: row threads of a group, a multiple of 32 up to the ones that cover nv in one
// pass (fewer loop over the rows in passes; 32 walks each candidate's own rows)
bool proj_shape_valid(int nv, int groups, int rows) {
    return (groups == 1 || groups == 2 || groups == 4 || groups == 8) && rows >= 32 && rows % 32 == 0 &&
           rows <= proj_row_threads(nv) && rows * groups <= kProjMaxThreads;
}
bool proj_groups_valid(int nv, int groups) { return proj_shape_valid(nv, groups, proj_row_threads(nv)); }
size_t proj_smem_bytes(int nv, int nx, int ny, int groups, int rows) {
    ProjSmem L{(nv + 3) / 4, rows * groups, std::max(nx, ny), groups};
    return L.bytes();
}
size_t proj_smem_bytes(int nv, int nx, int ny, int groups) {
    return proj_smem_bytes(nv, nx, ny, groups, proj_row_threads(nv));
}
int proj_group_width() { return kTU; }
int proj_max_lines() { return kMaxLines; }


size_t proj_staged_smem_bytes(int nv, int nx, int ny, int xstride, int groups, int rows, int slots) {
    StagedSmem L{(nv + 3) / 4, rows * groups, std::max(nx, ny), groups, slots, xstride};
    return L.bytes();
}
// Slots per stage buffer: 1 .. 64, and one buffer's bytes within an mbarrier phase's
// transaction count (< 2^20).
bool proj_slots_valid(int xstride, int slots) {
    return slots >= 1 && slots <= 64 && (size_t)slots * xstride * 4 < (1u << 20);
}

cudaError_t launch_proj_staged(int method, int groups, int rows, int slots, const Geom &g, const View *views,
                               const float *xs, const float *ampv, const uint8_t *map, void *proj, int out_dtype,
                               int vb, int vs, int vc, float margin, int *err, cudaStream_t st) {
    if (!proj_shape_valid(g.nv, groups, rows) || !proj_slots_valid(g.xstride, slots) ||
        g.xstride % 4 != 0 || g.xstride < g.nz + 2 || reinterpret_cast<uintptr_t>(xs) % 16 != 0)
        return cudaErrorInvalidValue;
    const size_t sm = proj_staged_smem_bytes(g.nv, g.nx, g.ny, g.xstride, groups, rows, slots);
    const int ngx = (g.nu + kTU - 1) / kTU;
    const int nblocks = ngx * vc;
    const int nt = rows * groups;
#define CTSIM_PROJ_STAGED_CASE(M, GR)                                                                 \
    if (method == M && groups == GR) {                                                                \
        cudaError_t e = allow_dynamic_smem((const void *)proj_staged_kernel<M, GR>, sm);              \
        if (e != cudaSuccess) return e;                                                               \
        proj_staged_kernel<M, GR><<<nblocks, nt, sm, st>>>(g, views, xs, ampv, map, proj, out_dtype, vb, vs,    \
                                                           margin, slots, err, ngx, vc);              \
        return cudaGetLastError();                                                                    \
    }
    CTSIM_PROJ_STAGED_CASE(kDD, 1) CTSIM_PROJ_STAGED_CASE(kDD, 2) CTSIM_PROJ_STAGED_CASE(kDD, 4)
    CTSIM_PROJ_STAGED_CASE(kDD, 8) CTSIM_PROJ_STAGED_CASE(kTF, 1) CTSIM_PROJ_STAGED_CASE(kTF, 2)
    CTSIM_PROJ_STAGED_CASE(kTF, 4) CTSIM_PROJ_STAGED_CASE(kTF, 8)
#undef CTSIM_PROJ_STAGED_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_proj(int method, int groups, int rows, bool pairs, const Geom &g, const View *views,
                        const float *xc, const float *ampv, const uint8_t *map, void *proj, int out_dtype, int vb,
                        int vs, int vc, float margin, cudaStream_t st) {
    if (!proj_shape_valid(g.nv, groups, rows)) return cudaErrorInvalidValue;
    const size_t sm = proj_smem_bytes(g.nv, g.nx, g.ny, groups, rows);
    const int ngx = (g.nu + kTU - 1) / kTU;
    const int nblocks = ngx * vc;
    // one thread per 4 detector rows (rows threads per group, more rows loop), groups
    // of those threads share the candidates
    const int nt = rows * groups;
#define CTSIM_PROJ_CASE(M, GR, P)                                                                     \
    if (method == M && groups == GR && pairs == P) {                                                  \
        cudaError_t e = allow_dynamic_smem((const void *)proj_kernel<M, GR, P>, sm);                  \
        if (e != cudaSuccess) return e;                                                               \
        proj_kernel<M, GR, P><<<nblocks, nt, sm, st>>>(g, views, xc, ampv, map, proj, out_dtype, vb, vs, margin, \
                                                       ngx, vc);                                      \
        return cudaGetLastError();                                                                    \
    }
    CTSIM_PROJ_CASE(kDD, 1, false) CTSIM_PROJ_CASE(kDD, 2, false) CTSIM_PROJ_CASE(kDD, 4, false)
    CTSIM_PROJ_CASE(kDD, 8, false) CTSIM_PROJ_CASE(kTF, 1, false) CTSIM_PROJ_CASE(kTF, 2, false)
    CTSIM_PROJ_CASE(kTF, 4, false) CTSIM_PROJ_CASE(kTF, 8, false)
    CTSIM_PROJ_CASE(kDD, 1, true) CTSIM_PROJ_CASE(kDD, 2, true) CTSIM_PROJ_CASE(kDD, 4, true)
    CTSIM_PROJ_CASE(kDD, 8, true) CTSIM_PROJ_CASE(kTF, 1, true) CTSIM_PROJ_CASE(kTF, 2, true)
    CTSIM_PROJ_CASE(kTF, 4, true) CTSIM_PROJ_CASE(kTF, 8, true)
#undef CTSIM_PROJ_CASE
    return cudaErrorInvalidValue;
}

template <int MODE, int MZ>
static cudaError_t launch_pd_mz(const Geom &g, const View *views, const void *proj, int in_dtype, const uint8_t *map,
                                void *image, int out_dtype, int vb, int vs, int vc, float scale, bool accumulate,
                                cudaStream_t st) {
    const int blocks = g.ny * ((g.nx + 7) / 8);
    if (accumulate)
        pd_kernel<MODE, MZ, true><<<blocks, 256, 0, st>>>(g, views, proj, map, image, out_dtype, vb, vs, vc, scale);
    else if (in_dtype == kBF16)
        pd_kernel<MODE, MZ, false, kBF16><<<blocks, 256, 0, st>>>(g, views, proj, map, image, out_dtype, vb, vs, vc,
                                                                  scale);
    else if (in_dtype == kF16)
        pd_kernel<MODE, MZ, false, kF16><<<blocks, 256, 0, st>>>(g, views, proj, map, image, out_dtype, vb, vs, vc,
                                                                 scale);
    else
        pd_kernel<MODE, MZ><<<blocks, 256, 0, st>>>(g, views, proj, map, image, out_dtype, vb, vs, vc, scale);
    return cudaGetLastError();
}

cudaError_t launch_pd(int mode, int mz, const Geom &g, const View *views, const void *proj, const uint8_t *map,
                      void *image, int out_dtype, int vb, int vs, int vc, float scale, cudaStream_t st,
                      bool accumulate, int in_dtype) {
    if (accumulate && (out_dtype != kF32 || scale != 1.0f || in_dtype != kF32)) return cudaErrorInvalidValue;
    if (in_dtype != kF32 && in_dtype != kBF16 && in_dtype != kF16) return cudaErrorInvalidValue;
#define CTSIM_PD_CASE(O, Z)                                                                                    \
    if (mode == O && mz == Z)                                                                                  \
        return launch_pd_mz<O, Z>(g, views, proj, in_dtype, map, image, out_dtype, vb, vs, vc, scale, accumulate, \
                                  st);
    CTSIM_PD_CASE(kPdOff, 1) CTSIM_PD_CASE(kPdOff, 2) CTSIM_PD_CASE(kPdOff, 4) CTSIM_PD_CASE(kPdOff, 8)
    CTSIM_PD_CASE(kPdClamp, 1) CTSIM_PD_CASE(kPdClamp, 2) CTSIM_PD_CASE(kPdClamp, 4) CTSIM_PD_CASE(kPdClamp, 8)
    CTSIM_PD_CASE(kPdVar, 1) CTSIM_PD_CASE(kPdVar, 2) CTSIM_PD_CASE(kPdVar, 4) CTSIM_PD_CASE(kPdVar, 8)
#undef CTSIM_PD_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_scale(float *y, size_t n, float s, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    scale_kernel<<<blocks, 256, 0, st>>>(y, n, s);
    return cudaGetLastError();
}

// A^T reading the unscaled sinogram (axial amplitude applied on the fly); used by the
// entry point that allocates nothing (noalloc.cu).
template <int METHOD, int MZ>
static cudaError_t launch_back_unscaled_mz(const Geom &g, const View *views, const float *proj, const float *ampv,
                                           const uint8_t *map, float *image, int vc, int qcap, int *err,
                                           cudaStream_t st) {
    const int blocks = g.ny * ((g.nx + 7) / 8);
    const size_t sm = back_smem_bytes(qcap);
    auto kfn = back_kernel<METHOD, MZ, false, kSrcF32>;
    cudaError_t e = allow_dynamic_smem((const void *)kfn, sm);
    if (e != cudaSuccess) return e;
    kfn<<<blocks, 256, sm, st>>>(g, views, proj, map, image, kF32, 0, 1, vc, 1.0f, qcap, err, ampv, 0);
    return cudaGetLastError();
}

cudaError_t launch_back_unscaled(int mz, const Geom &g, const View *views, const float *proj, const float *ampv,
                                 const uint8_t *map, float *image, int vc, int qcap, int *err, cudaStream_t st) {
    switch (mz) {
    case 1: return launch_back_unscaled_mz<kDD, 1>(g, views, proj, ampv, map, image, vc, qcap, err, st);
    case 2: return launch_back_unscaled_mz<kDD, 2>(g, views, proj, ampv, map, image, vc, qcap, err, st);
    case 4: return launch_back_unscaled_mz<kDD, 4>(g, views, proj, ampv, map, image, vc, qcap, err, st);
    case 8: return launch_back_unscaled_mz<kDD, 8>(g, views, proj, ampv, map, image, vc, qcap, err, st);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Batched launches.  One persistent grid (the resident blocks of the whole GPU) walks
// the flat block list of up to kBatchMax tasks -- plans of different geometries -- and
// runs each block's work with its task's tables; the task table is a __grid_constant__
// kernel parameter, so a batch needs no device allocation and can be graph-captured.
// ---------------------------------------------------------------------------
// LOWP: outputs in each task's storage type; otherwise FP32 (a compile-time store).
template <int METHOD, int GROUPS, bool PAIRS, bool LOWP>
__global__ void __launch_bounds__(kProjMaxThreads) proj_batch_kernel(const __grid_constant__ ProjBatch b) {
    extern __shared__ float4 acc4_batch[];
    for (int blk = blockIdx.x; blk < b.total; blk += gridDim.x) {
        int lo = 0, hi = b.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b.t[mid].first <= blk) lo = mid; else hi = mid - 1;
        }
        const ProjTask &T = b.t[lo];
        int bx, by;
        view_grouped_block(blk - T.first, T.gx, T.vc, bx, by);
        proj_block<METHOD, GROUPS, PAIRS>(T.g, T.views, T.xs, T.ampv, T.map, T.proj, LOWP ? T.out_dtype : kF32, T.vb,
                                          T.vs, T.margin, acc4_batch, bx, by);
        __syncthreads();  // the next block reuses the shared accumulators
    }
}

// The staged forward projector over the flat blocks of many plans (same group count,
// row threads and slots; each task its own geometry and scratch); the mbarriers and their
// phases persist across the items of a block.
template <int METHOD, int GROUPS, bool LOWP>
__global__ void __launch_bounds__(kProjMaxThreads, 3) proj_staged_batch_kernel(const __grid_constant__ ProjBatch b,
                                                                               int slots) {
    extern __shared__ float4 smem_staged_batch[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_staged_batch);
    staged_bars_init(bar);
    unsigned phase = kStagedPhase0;
    for (int blk = blockIdx.x; blk < b.total; blk += gridDim.x) {
        int lo = 0, hi = b.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b.t[mid].first <= blk) lo = mid; else hi = mid - 1;
        }
        const ProjTask &T = b.t[lo];
        int bx, by;
        view_grouped_block(blk - T.first, T.gx, T.vc, bx, by);
        if (!proj_staged_block<METHOD, GROUPS>(T.g, T.views, T.xs, T.ampv, T.map, T.proj, LOWP ? T.out_dtype : kF32,
                                               T.vb, T.vs, T.margin, slots, T.err, smem_staged_batch + 2, bar, phase,
                                               bx, by))
            return;
        __syncthreads();  // the next item reuses the shared accumulators and tables
    }
}

template <int METHOD, int MZ, bool VEC, bool LOWP, int SRC>
__global__ void __launch_bounds__(256) back_batch_kernel(const __grid_constant__ BackBatch b) {
    extern __shared__ float smem_batch[];
    for (int blk = blockIdx.x; blk < b.total; blk += gridDim.x) {
        int lo = 0, hi = b.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b.t[mid].first <= blk) lo = mid; else hi = mid - 1;
        }
        const BackTask &T = b.t[lo];
        back_block<METHOD, MZ, VEC, SRC>(T.g, T.views, T.ps, T.map, T.image, LOWP ? T.out_dtype : kF32, T.vb, T.vs,
                                         T.vc, T.scale, T.qcap, T.err, T.ampv, smem_batch, blk - T.first);
        // the per-warp row buffers are laid out with the task's own stride, so a warp may
        // not start the next item (possibly another task) while its neighbours still work
        __syncthreads();
    }
}

int proj_task_blocks(const Geom &g, int view_count) { return ((g.nu + kTU - 1) / kTU) * view_count; }
int back_task_blocks(const Geom &g) { return g.ny * ((g.nx + 7) / 8); }
int proj_row_threads_of(int nv) { return proj_row_threads(nv); }

template <class K>
static int persistent_grid(K kernel, int threads, size_t smem, int total) {
    int dev = 0, sms = 148, per_sm = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return std::max(1, std::min(total, sms * per_sm));
}

cudaError_t launch_proj_batch(int method, int groups, int row_threads, bool pairs, bool lowp, size_t smem,
                              const ProjBatch &b, cudaStream_t st) {
    if (b.n < 1 || b.total < 1) return cudaSuccess;
    const int nt = row_threads * groups;
#define CTSIM_PB_CASE(M, GR)                                                                          \
    if (method == M && groups == GR) {                                                                \
        auto k = pairs ? (lowp ? proj_batch_kernel<M, GR, true, true> : proj_batch_kernel<M, GR, true, false>) \
                       : (lowp ? proj_batch_kernel<M, GR, false, true> : proj_batch_kernel<M, GR, false, false>); \
        cudaError_t e = allow_dynamic_smem((const void *)k, smem);                                    \
        if (e != cudaSuccess) return e;                                                               \
        k<<<persistent_grid(k, nt, smem, b.total), nt, smem, st>>>(b);                                \
        return cudaGetLastError();                                                                    \
    }
    CTSIM_PB_CASE(kDD, 1) CTSIM_PB_CASE(kDD, 2) CTSIM_PB_CASE(kDD, 4) CTSIM_PB_CASE(kDD, 8)
    CTSIM_PB_CASE(kTF, 1) CTSIM_PB_CASE(kTF, 2) CTSIM_PB_CASE(kTF, 4) CTSIM_PB_CASE(kTF, 8)
#undef CTSIM_PB_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_proj_staged_batch(int method, int groups, int row_threads, int slots, bool lowp, size_t smem,
                                     const ProjBatch &b, cudaStream_t st) {
    if (b.n < 1 || b.total < 1) return cudaSuccess;
    const int nt = row_threads * groups;
#define CTSIM_PSB_CASE(M, GR)                                                                         \
    if (method == M && groups == GR) {                                                                \
        auto k = lowp ? proj_staged_batch_kernel<M, GR, true> : proj_staged_batch_kernel<M, GR, false>; \
        cudaError_t e = allow_dynamic_smem((const void *)k, smem);                                    \
        if (e != cudaSuccess) return e;                                                               \
        k<<<persistent_grid(k, nt, smem, b.total), nt, smem, st>>>(b, slots);                         \
        return cudaGetLastError();                                                                    \
    }
    CTSIM_PSB_CASE(kDD, 1) CTSIM_PSB_CASE(kDD, 2) CTSIM_PSB_CASE(kDD, 4) CTSIM_PSB_CASE(kDD, 8)
    CTSIM_PSB_CASE(kTF, 1) CTSIM_PSB_CASE(kTF, 2) CTSIM_PSB_CASE(kTF, 4) CTSIM_PSB_CASE(kTF, 8)
#undef CTSIM_PSB_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_back_batch(int method, int mz, bool vec, bool lowp, size_t smem, const BackBatch &b,
                              cudaStream_t st, int src) {
    if (b.n < 1 || b.total < 1) return cudaSuccess;
    if (src != kSrcScaled && src != kSrcBF16 && src != kSrcF16) return cudaErrorInvalidValue;
#define CTSIM_BB_LAUNCH(M, Z, V, S)                                                                   \
    {                                                                                                 \
        auto k = lowp ? back_batch_kernel<M, Z, V, true, S> : back_batch_kernel<M, Z, V, false, S>;   \
        cudaError_t e = allow_dynamic_smem((const void *)k, smem);                                    \
        if (e != cudaSuccess) return e;                                                               \
        k<<<persistent_grid(k, 256, smem, b.total), 256, smem, st>>>(b);                              \
        return cudaGetLastError();                                                                    \
    }
#define CTSIM_BB_CASE(M, Z, V)                                                                        \
    if (method == M && mz == Z && vec == V) {                                                         \
        if (src == kSrcBF16) CTSIM_BB_LAUNCH(M, Z, V, kSrcBF16)                                       \
        if (src == kSrcF16) CTSIM_BB_LAUNCH(M, Z, V, kSrcF16)                                         \
        CTSIM_BB_LAUNCH(M, Z, V, kSrcScaled)                                                          \
    }
    CTSIM_BB_CASE(kDD, 1, true) CTSIM_BB_CASE(kDD, 2, true) CTSIM_BB_CASE(kDD, 4, true) CTSIM_BB_CASE(kDD, 8, true)
    CTSIM_BB_CASE(kDD, 1, false) CTSIM_BB_CASE(kDD, 2, false) CTSIM_BB_CASE(kDD, 4, false) CTSIM_BB_CASE(kDD, 8, false)
    CTSIM_BB_CASE(kTF, 1, true) CTSIM_BB_CASE(kTF, 2, true) CTSIM_BB_CASE(kTF, 4, true) CTSIM_BB_CASE(kTF, 8, true)
    CTSIM_BB_CASE(kTF, 1, false) CTSIM_BB_CASE(kTF, 2, false) CTSIM_BB_CASE(kTF, 4, false) CTSIM_BB_CASE(kTF, 8, false)
#undef CTSIM_BB_CASE
#undef CTSIM_BB_LAUNCH
    return cudaErrorInvalidValue;
}

}  // namespace ctsim
