// Launcher declarations for the projector kernels (kernels.cu).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace ctsim {

// ps = proj (any storage type) * ampv (ampv may be null: plain conversion to FP32)
cudaError_t launch_prescale(const void *proj, int in_dtype, const float *ampv, float *ps, size_t nuv, size_t n,
                            cudaStream_t st);

// Sinogram sources of the backprojector: FP32 already multiplied by the axial amplitude
// ampv (a pre-scaled copy, or a residual written that way), or the stored sinogram in
// FP32, BF16 or FP16, multiplied by ampv as it is read.  launch_back and the batches take
// kSrcScaled, kSrcBF16 and kSrcF16 (kSrcF32 serves the entry point without allocations).
enum BackSrc { kSrcScaled = 0, kSrcF32 = 1, kSrcBF16 = 2, kSrcF16 = 3 };
cudaError_t launch_back(int method, int mz, const Geom &g, const View *views, const void *ps, const uint8_t *map,
                        void *image, int out_dtype, int view_begin, int view_stride, int view_count, float scale,
                        int qcap, int *err, cudaStream_t st, bool accumulate = false, int y_begin = 0,
                        int y_end = -1, int src = kSrcScaled, const float *ampv = nullptr);
size_t back_smem_bytes(int qcap);
cudaError_t launch_back_unscaled(int mz, const Geom &g, const View *views, const float *proj, const float *ampv,
                                 const uint8_t *map, float *image, int view_count, int qcap, int *err,
                                 cudaStream_t st);

// pairs: the (X, slope) layout of the column prefix sums (forward_pairs below)
cudaError_t launch_prefix(const void *image, int in_dtype, float *xs, int nxy, int nz, bool pairs, int xstride,
                          cudaStream_t st);

cudaError_t launch_proj(int method, int groups, int rows, bool pairs, const Geom &g, const View *views,
                        const float *xs, const float *ampv, const uint8_t *map, void *proj, int out_dtype,
                        int view_begin, int view_stride, int view_count, float margin, cudaStream_t st);
// The paired prefix layout when it is small enough to stay cache-resident (<= 160 MB).
inline bool forward_pairs(long long nxy, int nz) { return 8LL * nxy * (nz + 1) <= 160LL * 1024 * 1024; }
int proj_default_groups(int nv);
int proj_default_rows(int nv);
bool proj_groups_valid(int nv, int groups);
bool proj_shape_valid(int nv, int groups, int rows);
size_t proj_smem_bytes(int nv, int nx, int ny, int groups, int rows);
// The forward projector with each candidate's prefix column staged in shared memory by
// bulk copies (plain layout, g.xstride a multiple of 4 and >= nz + 2, xs 16-byte aligned):
// `slots` columns per stage buffer, two buffers.  A stage wait that runs out sets bit 4
// of *err.
cudaError_t launch_proj_staged(int method, int groups, int rows, int slots, const Geom &g, const View *views,
                               const float *xs, const float *ampv, const uint8_t *map, void *proj, int out_dtype,
                               int view_begin, int view_stride, int view_count, float margin, int *err,
                               cudaStream_t st);
size_t proj_staged_smem_bytes(int nv, int nx, int ny, int xstride, int groups, int rows, int slots);
bool proj_slots_valid(int xstride, int slots);

// voxel-driven bilinear modes: back,pd (v outside the detector skipped), back,hpd (v
// clamped), back,var (geom/cbct/cbct_back_var.c)
enum PdMode { kPdOff = 0, kPdClamp = 1, kPdVar = 2 };
// proj in storage type in_dtype (kF32, kBF16, kF16), read as it is.
cudaError_t launch_pd(int mode, int mz, const Geom &g, const View *views, const void *proj,
                      const uint8_t *map, void *image, int out_dtype, int view_begin, int view_stride,
                      int view_count, float scale, cudaStream_t st, bool accumulate = false, int in_dtype = kF32);

cudaError_t launch_scale(float *y, size_t n, float s, cudaStream_t st);

// ---------------------------------------------------------------------------
// Batched launches: the blocks of many plans' A (or A^T) in one persistent grid.
// ---------------------------------------------------------------------------
constexpr int kBatchMax = 64;  // tasks per launch (the task table travels as a kernel parameter)

struct ProjTask {
    Geom g;
    const View *views;
    const float *xs;
    const float *ampv;
    const uint8_t *map;
    void *proj;
    int out_dtype;
    int vb, vs, vc, gx, first;  // view selection, blocks along u, first flat block of the task
    float margin;
    int *err;               // the plan's error flag (staged projector: a stage wait that ran out)
};
struct ProjBatch {
    int n, total;  // tasks, flat blocks of all tasks
    ProjTask t[kBatchMax];
};

struct BackTask {
    Geom g;
    const View *views;
    const void *ps;         // the class's source form (BackSrc)
    const float *ampv;      // the plan's axial amplitudes (unscaled sources)
    const uint8_t *map;
    void *image;
    int out_dtype;
    int *err;
    int vb, vs, vc, qcap, first;
    float scale;
};
struct BackBatch {
    int n, total;
    BackTask t[kBatchMax];
};

// The flat blocks of a task: A (u groups x views), A^T (rows x column tiles).
int proj_task_blocks(const Geom &g, int view_count);
int back_task_blocks(const Geom &g);
int proj_row_threads_of(int nv);
// lowp: some task stores BF16/FP16 (each task's out_dtype); otherwise all store FP32
cudaError_t launch_proj_batch(int method, int groups, int row_threads, bool pairs, bool lowp, size_t smem,
                              const ProjBatch &b, cudaStream_t st);
cudaError_t launch_back_batch(int method, int mz, bool vec, bool lowp, size_t smem, const BackBatch &b,
                              cudaStream_t st, int src = kSrcScaled);
// The staged forward projector (launch_proj_staged) over a batch of plain-layout plans.
cudaError_t launch_proj_staged_batch(int method, int groups, int row_threads, int slots, bool lowp, size_t smem,
                                     const ProjBatch &b, cudaStream_t st);

// Raises (never lowers) a kernel's dynamic shared-memory limit on the current device.
cudaError_t allow_dynamic_smem(const void *kfn, size_t bytes);

size_t proj_smem_bytes(int nv, int nx, int ny, int groups);
int proj_group_width();
int proj_max_lines();

}  // namespace ctsim
