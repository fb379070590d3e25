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

namespace ctsim {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// A^T: one warp per voxel column, lanes along z; 8 columns (consecutive ix) per block.
// For each view the warp forms the u-weighted detector column
//     Q[iv] = sum_iu w_u(iu) * (proj[iu][iv] * ampv[iu][iv])
// over the rows the column's voxels can touch, in shared memory, then every lane
// gathers its voxels' axial footprints from Q with the reference's exact weights
// (geom/cbct/cbct_back.c:316-359).  Accumulation over views stays in registers.
// ---------------------------------------------------------------------------
template <int METHOD, int MZ>
__global__ void __launch_bounds__(256) back_kernel(Geom g, const View *__restrict__ views,
                                                   const float *__restrict__ proj, const float *__restrict__ ampv,
                                                   const uint8_t *__restrict__ map, float *__restrict__ image,
                                                   int view_begin, int view_stride, int view_count, float scale,
                                                   int qcap, int *__restrict__ err) {
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *Q = smem + warp * qcap;
    const int tiles_x = (g.nx + 7) >> 3;
    const int iy = blockIdx.x / tiles_x;
    const int ix = (blockIdx.x % tiles_x) * 8 + warp;
    if (ix >= g.nx || iy >= g.ny) return;
    const size_t nxy = (size_t)g.nx * g.ny;
    const size_t nuv = (size_t)g.nu * g.nv;
    const bool on = map[iy * g.nx + ix] != 0;
    const int zpass = 32 * MZ;
    for (int iz0 = 0; iz0 < g.nz; iz0 += zpass) {
        const int izn = min(zpass, g.nz - iz0);
        float acc[MZ];
#pragma unroll
        for (int m = 0; m < MZ; m++) acc[m] = 0.0f;
        if (on) {
            for (int k0 = 0; k0 < view_count; k0 += 32) {
                ColumnFP my;
                my.hit = false;
                const int kl = k0 + lane;
                if (kl < view_count) my = column_footprint<METHOD>(g, views[view_begin + kl * view_stride], ix, iy);
                const int nk = min(32, view_count - k0);
                for (int j = 0; j < nk; j++) {
                    if (!__shfl_sync(kFull, (int)my.hit, j)) continue;
                    const int iumin = __shfl_sync(kFull, my.iumin, j);
                    const int iumax = __shfl_sync(kFull, my.iumax, j);
                    const float p0 = __shfl_sync(kFull, my.p0, j), p1 = __shfl_sync(kFull, my.p1, j);
                    float p2 = 0.f, p3 = 0.f;
                    if (METHOD == kTF) { p2 = __shfl_sync(kFull, my.p2, j); p3 = __shfl_sync(kFull, my.p3, j); }
                    const float ampu = __shfl_sync(kFull, my.ampu, j);
                    const float zinc = __shfl_sync(kFull, my.zinc, j);
                    const float vstart = __shfl_sync(kFull, my.vstart, j);
                    // rows reachable by voxels [iz0, iz0+izn): monotone in iz
                    float a0, b0, a1, b1;
                    voxel_v_extent(g, vstart, zinc, iz0, a0, b0);
                    voxel_v_extent(g, vstart, zinc, iz0 + izn - 1, a1, b1);
                    if (!(a0 < (float)g.nv)) continue;  // whole pass above the detector
                    const int r_lo = (int)floorf(a0);
                    int r_hi = min((int)floorf(b1), g.nv - 1);
                    if (r_lo > r_hi) continue;
                    if (r_hi - r_lo + 1 > qcap) {
                        if (lane == 0) atomicOr(err, 1);
                        r_hi = r_lo + qcap - 1;
                    }
                    const int nb = iumax - iumin + 1;
                    const float wl = lane < nb ? u_weight<METHOD>(iumin + lane, iumin, iumax, p0, p1, p2, p3) : 0.0f;
                    const float *pv = proj + (size_t)(k0 + j) * nuv + (size_t)iumin * g.nv;
                    const float *av = ampv + (size_t)iumin * g.nv;
                    for (int rb = r_lo; rb <= r_hi; rb += 32) {
                        const int r = rb + lane;
                        const bool ok = r <= r_hi;
                        float q = 0.0f;
                        for (int b = 0; b < nb; b++) {
                            const float w = __shfl_sync(kFull, wl, b);
                            if (ok) {
                                const size_t o = (size_t)b * g.nv + r;
                                q = fmaf(__ldg(pv + o) * __ldg(av + o), w, q);
                            }
                        }
                        if (ok) Q[r - r_lo] = q;
                    }
                    __syncwarp();
#pragma unroll
                    for (int m = 0; m < MZ; m++) {
                        const int dz = lane + 32 * m;
                        if (dz < izn) {
                            float vmin, vmax;
                            voxel_v_extent(g, vstart, zinc, iz0 + dz, vmin, vmax);
                            if (!(vmin > vmax)) {
                                const int lo = (int)floorf(vmin);
                                const int hi = min(min(min((int)floorf(vmax), g.nv - 1), lo + kMaxRowsV - 1), r_hi);
                                if (lo <= hi) {
                                    float val;
                                    if (lo == hi) {
                                        val = fsub(vmax, vmin) * Q[lo - r_lo];
                                    } else {
                                        val = fsub((float)(lo + 1), vmin) * Q[lo - r_lo];
                                        for (int r = lo + 1; r < hi; r++) val += Q[r - r_lo];
                                        val = fmaf(fsub(vmax, (float)hi), Q[hi - r_lo], val);
                                    }
                                    acc[m] = fmaf(ampu, val, acc[m]);
                                }
                            }
                        }
                    }
                    __syncwarp();
                }
            }
        }
#pragma unroll
        for (int m = 0; m < MZ; m++) {
            const int dz = lane + 32 * m;
            if (dz < izn) image[(size_t)(iz0 + dz) * nxy + (size_t)iy * g.nx + ix] = on ? acc[m] * scale : 0.0f;
        }
    }
}

// ---------------------------------------------------------------------------
// Axial prefix sums of every voxel column (input of the forward projector):
//   xc[col*(nz+1) + k] = sum_{j<k} image[j][col],  col = iy*nx + ix.
// 32 columns per block; a 32x32 tile is transposed through shared memory so that
// both the image reads and the prefix writes are coalesced.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) prefix_kernel(const float *__restrict__ image, float *__restrict__ xc, int nxy,
                                                     int nz) {
    __shared__ float tile[32][33];
    __shared__ float carry[32];
    const int c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    if (threadIdx.x < 32) carry[threadIdx.x] = 0.0f;
    const size_t stride = (size_t)nz + 1;
    for (int z0 = 0; z0 < nz; z0 += 32) {
        __syncthreads();
        for (int zz = ty; zz < 32; zz += 8) {
            const int z = z0 + zz, c = c0 + tx;
            tile[zz][tx] = (z < nz && c < nxy) ? image[(size_t)z * nxy + c] : 0.0f;
        }
        __syncthreads();
        // warp ty scans columns ty, ty+8, ty+16, ty+24 along z (lane = z)
        for (int cc = ty; cc < 32; cc += 8) {
            float v = tile[tx][cc];
            // sequential-order inclusive scan (Hillis-Steele gives the same rounding for all columns)
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float n = __shfl_up_sync(kFull, v, o);
                if (tx >= o) v += n;
            }
            const float base = carry[cc];
            const int c = c0 + cc, z = z0 + tx;
            if (c < nxy && z < nz) xc[(size_t)c * stride + z + 1] = base + v;
            const float tot = __shfl_sync(kFull, v, 31);
            __syncwarp();
            if (tx == 0) carry[cc] = base + tot;
        }
    }
    if (threadIdx.x < 32 && c0 + threadIdx.x < nxy) xc[(size_t)(c0 + threadIdx.x) * stride] = 0.0f;
}

// ---------------------------------------------------------------------------
// A: one block per (group of kTU detector columns, view).  Candidate voxel columns
// are enumerated line by line (lines across the ray direction; the projected
// column centre is monotone along a line, so the candidates of a line form one
// interval found by binary search).  Each candidate's footprint is evaluated
// exactly; a thread owns detector rows and adds
//     w_u(iu) * ampu * zinc * (X(iv+1) - X(iv))
// where X is the linear interpolation of the column's axial prefix sums at the
// row boundaries -- the integral form of the distance-driven axial weights
// (geom/cbct/cbct_proj.c:382-420).  Accumulators are thread-private shared-memory
// cells: no atomics, deterministic.
// ---------------------------------------------------------------------------
constexpr int kTU = 8;
constexpr int kProjThreads = 256;
constexpr int kMaxLines = 2048;

template <int METHOD>
__global__ void __launch_bounds__(kProjThreads) proj_kernel(Geom g, const View *__restrict__ views,
                                                            const float *__restrict__ xc,
                                                            const float *__restrict__ ampv,
                                                            const uint8_t *__restrict__ map, float *__restrict__ proj,
                                                            int view_begin, int view_stride, float margin) {
    extern __shared__ float acc_s[];  // [kTU][nv]
    __shared__ int line_start[kMaxLines];
    __shared__ int line_off[kMaxLines + 1];
    __shared__ int s_col[kProjThreads];
    __shared__ float s_b0[kProjThreads], s_iz[kProjThreads];
    __shared__ int s_rlo[kProjThreads], s_rhi[kProjThreads], s_j[kProjThreads];
    __shared__ float s_w[kProjThreads][kTU];
    __shared__ int s_warp_tot[kProjThreads / 32];

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int iu0 = blockIdx.x * kTU;
    const int k = blockIdx.y;
    const View v = views[view_begin + k * view_stride];
    const int nv = g.nv;
    for (int i = t; i < kTU * nv; i += kProjThreads) acc_s[i] = 0.0f;

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
        const float r = tp / ds;
        return (g.det == 1 ? g.sdd_du * r : g.sdd_du * atanf(r)) - g.wu + 0.5f;
    };

    // 1. candidate interval of every line
    int my_count_total = 0;
    for (int L = t; L < nlines; L += kProjThreads) {
        auto f = [&](int p) { return rows ? centre_u(p, L) : centre_u(L, p); };
        const float fa = f(0), fb = f(npos - 1);
        const bool inc = fb >= fa;
        // first position with f inside [ulo, uhi] and last one (f monotone)
        int lo = 0, hi = npos;  // lower bound of "not before the window"
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float fm = f(mid);
            const bool before = inc ? (fm < ulo) : (fm > uhi);
            if (before) lo = mid + 1; else hi = mid;
        }
        const int first = lo;
        lo = first; hi = npos;  // first position beyond the window
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const float fm = f(mid);
            const bool beyond = inc ? (fm > uhi) : (fm < ulo);
            if (beyond) hi = mid; else lo = mid + 1;
        }
        line_start[L] = first;
        line_off[L] = lo - first;  // count, turned into offsets below
    }
    __syncthreads();
    // 2. exclusive scan of the counts (lines <= kMaxLines)
    {
        const int per = (nlines + kProjThreads - 1) / kProjThreads;
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
        if (t == kProjThreads - 1) line_off[nlines] = run;
        my_count_total = 0;
    }
    __syncthreads();
    const int ncand = line_off[nlines];
    const size_t zstride = (size_t)g.nz + 1;
    const float fnz = (float)g.nz;

    for (int c0 = 0; c0 < ncand; c0 += kProjThreads) {
        // 3. footprints of this chunk of candidates
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
                            s_w[t][j] = w;
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
        // 4. accumulate rows
        const int nslot = min(kProjThreads, ncand - c0);
        for (int s = 0; s < nslot; s++) {
            const int jj = s_j[s];
            if (jj < 0) continue;
            const int rlo = s_rlo[s], rhi = s_rhi[s];
            const float b0 = s_b0[s], iz = s_iz[s];
            const float *x = xc + (size_t)s_col[s] * zstride;
            const int jlo = jj & 0xff, jhi = jj >> 8;
            for (int rbase = warp * 32; rbase < nv; rbase += kProjThreads) {
                if (rbase > rhi || rbase + 31 < rlo) continue;  // warp-uniform
                const int iv = rbase + lane;
                // X at the row's two boundaries
                float sl = fminf(fmaxf(((float)iv - b0) * iz, 0.0f), fnz);
                float sh = fminf(fmaxf(((float)(iv + 1) - b0) * iz, 0.0f), fnz);
                int kl = min((int)sl, g.nz - 1), kh = min((int)sh, g.nz - 1);
                const float xl0 = __ldg(x + kl), xl1 = __ldg(x + kl + 1);
                const float xh0 = __ldg(x + kh), xh1 = __ldg(x + kh + 1);
                const float Xl = fmaf(sl - (float)kl, xl1 - xl0, xl0);
                const float Xh = fmaf(sh - (float)kh, xh1 - xh0, xh0);
                const float R = Xh - Xl;
                if (iv < nv && iv >= rlo && iv <= rhi) {
                    for (int j = jlo; j <= jhi; j++) acc_s[j * nv + iv] = fmaf(s_w[s][j], R, acc_s[j * nv + iv]);
                }
            }
        }
        __syncthreads();
    }
    // 5. axial amplitude and store
    float *out = proj + (size_t)k * g.nu * nv;
    for (int j = 0; j < kTU; j++) {
        const int iu = iu0 + j;
        if (iu >= g.nu) break;
        for (int iv = t; iv < nv; iv += kProjThreads)
            out[(size_t)iu * nv + iv] = acc_s[j * nv + iv] * ampv[(size_t)iu * nv + iv];
    }
    (void)my_count_total;
}

// ---------------------------------------------------------------------------
// FDK voxel-driven bilinear backprojection (geom/cbct/cbct_back.c:7-133): warp
// per column, lanes along z.  Per-view column quantities (u, w2, w2s) are computed
// by lane j for view k0+j and broadcast; every voxel accumulates the views in the
// reference's order with its exact float operations.
// ---------------------------------------------------------------------------
template <bool OFF, int MZ>
__global__ void __launch_bounds__(256) pd_kernel(Geom g, const View *__restrict__ views,
                                                 const float *__restrict__ proj, const uint8_t *__restrict__ map,
                                                 float *__restrict__ image, int view_begin, int view_stride,
                                                 int view_count, float scale) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (g.nx + 7) >> 3;
    const int iy = blockIdx.x / tiles_x;
    const int ix = (blockIdx.x % tiles_x) * 8 + warp;
    if (ix >= g.nx || iy >= g.ny) return;
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
            zc0[m] = fmul(fadd((float)(iz0 + lane + 32 * m), g.wz_pd), g.dz);
        }
        if (on) {
            for (int k0 = 0; k0 < view_count; k0 += 32) {
                float u = -1.0f, w2 = 0.0f, w2s = 0.0f, couch = 0.0f;
                const int kl = k0 + lane;
                if (kl < view_count) {
                    const View v = views[view_begin + kl * view_stride];
                    const float xr = fsub(fmul(xc, v.cos_a), fmul(yc, v.sin_a));
                    const float yr = fadd(fmul(xc, v.sin_a), fmul(yc, v.cos_a));
                    const float den = fadd(g.sad, yr);
                    if (g.det == 1) {
                        w2 = fdiv(g.sdd, den);
                        w2s = fmul(w2, w2);
                        u = fsub(fdiv(fmul(xr, w2), g.du), g.wu);
                    } else {
                        const float xo = fsub(xr, g.roff);
                        const double at = atan((double)fdiv(xo, den));
                        u = (float)__dsub_rn(__ddiv_rn(__dmul_rn(at, (double)g.sdd), (double)g.du), (double)g.wu);
                        w2s = fdiv(fmul(g.sdd, g.sdd), fadd(fmul(den, den), fmul(xo, xo)));
                        w2 = fdiv(g.sdd, den);
                    }
                    couch = v.couch_pd;
                }
                const int nk = min(32, view_count - k0);
                for (int j = 0; j < nk; j++) {
                    const float uj = __shfl_sync(kFull, u, j);
                    const float w2j = __shfl_sync(kFull, w2, j);
                    const float w2sj = __shfl_sync(kFull, w2s, j);
                    const float cj = __shfl_sync(kFull, couch, j);
                    if (uj < g.u_lo || uj > g.u_hi) continue;  // cbct_back.c:90
                    const int iu = (int)floorf(uj);
                    const float wul = fsub(uj, (float)iu);
                    const float *pv = proj + (size_t)(k0 + j) * nuv + (size_t)iu * g.nv;
#pragma unroll
                    for (int m = 0; m < MZ; m++) {
                        if (lane + 32 * m < izn) {
                            const float zc = fadd(zc0[m], cj);
                            float vv = fsub(fdiv(fmul(zc, w2j), g.dv), g.wv);
                            bool use = true;
                            if (OFF) {
                                use = !(vv < g.v_lo) && !(vv > g.v_hi);
                            } else {
                                vv = vv > 0.5f ? vv : 0.5f;
                                vv = vv < g.v_clamp_hi ? vv : g.v_clamp_hi;
                            }
                            if (use) {
                                const int iv = (int)floorf(vv);
                                const float wvl = fsub(vv, (float)iv);
                                const float omv = fsub(1.0f, wvl);
                                const float *p = pv + iv;
                                const float s0 = fadd(fmul(omv, __ldg(p)), fmul(wvl, __ldg(p + 1)));
                                const float s1 = fadd(fmul(omv, __ldg(p + g.nv)), fmul(wvl, __ldg(p + g.nv + 1)));
                                const float val = fadd(fmul(fsub(1.0f, wul), s0), fmul(wul, s1));
                                acc[m] = fadd(acc[m], fmul(w2sj, val));
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
                image[(size_t)(iz0 + dz) * nxy + (size_t)iy * g.nx + ix] = r;
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
template <int METHOD, int MZ>
static cudaError_t launch_back_mz(const Geom &g, const View *views, const float *proj, const float *ampv,
                                  const uint8_t *map, float *image, int vb, int vs, int vc, float scale, int qcap,
                                  int *err, cudaStream_t st) {
    const int blocks = g.ny * ((g.nx + 7) / 8);
    const size_t sm = (size_t)8 * qcap * sizeof(float);
    auto kfn = back_kernel<METHOD, MZ>;
    cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    kfn<<<blocks, 256, sm, st>>>(g, views, proj, ampv, map, image, vb, vs, vc, scale, qcap, err);
    return cudaGetLastError();
}

cudaError_t launch_back(int method, int mz, const Geom &g, const View *views, const float *proj, const float *ampv,
                        const uint8_t *map, float *image, int vb, int vs, int vc, float scale, int qcap, int *err,
                        cudaStream_t st) {
#define CTSIM_BACK_CASE(M, Z) \
    if (method == M && mz == Z) return launch_back_mz<M, Z>(g, views, proj, ampv, map, image, vb, vs, vc, scale, qcap, err, st);
    CTSIM_BACK_CASE(kDD, 1) CTSIM_BACK_CASE(kDD, 2) CTSIM_BACK_CASE(kDD, 4) CTSIM_BACK_CASE(kDD, 8)
    CTSIM_BACK_CASE(kTF, 1) CTSIM_BACK_CASE(kTF, 2) CTSIM_BACK_CASE(kTF, 4) CTSIM_BACK_CASE(kTF, 8)
#undef CTSIM_BACK_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_prefix(const float *image, float *xc, int nxy, int nz, cudaStream_t st) {
    const int blocks = (nxy + 31) / 32;
    prefix_kernel<<<blocks, 256, 0, st>>>(image, xc, nxy, nz);
    return cudaGetLastError();
}

size_t proj_smem_bytes(int nv) { return (size_t)kTU * nv * sizeof(float); }
int proj_group_width() { return kTU; }
int proj_max_lines() { return kMaxLines; }

cudaError_t launch_proj(int method, const Geom &g, const View *views, const float *xc, const float *ampv,
                        const uint8_t *map, float *proj, int vb, int vs, int vc, float margin, cudaStream_t st) {
    const size_t sm = proj_smem_bytes(g.nv);
    dim3 grid((g.nu + kTU - 1) / kTU, vc);
    if (method == kDD) {
        cudaError_t e = cudaFuncSetAttribute(proj_kernel<kDD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        proj_kernel<kDD><<<grid, kProjThreads, sm, st>>>(g, views, xc, ampv, map, proj, vb, vs, margin);
    } else {
        cudaError_t e = cudaFuncSetAttribute(proj_kernel<kTF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        proj_kernel<kTF><<<grid, kProjThreads, sm, st>>>(g, views, xc, ampv, map, proj, vb, vs, margin);
    }
    return cudaGetLastError();
}

template <bool OFF, int MZ>
static cudaError_t launch_pd_mz(const Geom &g, const View *views, const float *proj, const uint8_t *map,
                                float *image, int vb, int vs, int vc, float scale, cudaStream_t st) {
    const int blocks = g.ny * ((g.nx + 7) / 8);
    pd_kernel<OFF, MZ><<<blocks, 256, 0, st>>>(g, views, proj, map, image, vb, vs, vc, scale);
    return cudaGetLastError();
}

cudaError_t launch_pd(bool off, int mz, const Geom &g, const View *views, const float *proj, const uint8_t *map,
                      float *image, int vb, int vs, int vc, float scale, cudaStream_t st) {
#define CTSIM_PD_CASE(O, Z) \
    if (off == O && mz == Z) return launch_pd_mz<O, Z>(g, views, proj, map, image, vb, vs, vc, scale, st);
    CTSIM_PD_CASE(true, 1) CTSIM_PD_CASE(true, 2) CTSIM_PD_CASE(true, 4) CTSIM_PD_CASE(true, 8)
    CTSIM_PD_CASE(false, 1) CTSIM_PD_CASE(false, 2) CTSIM_PD_CASE(false, 4) CTSIM_PD_CASE(false, 8)
#undef CTSIM_PD_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_scale(float *y, size_t n, float s, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    scale_kernel<<<blocks, 256, 0, st>>>(y, n, s);
    return cudaGetLastError();
}

}  // namespace ctsim
