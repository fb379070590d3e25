/*
 * ctsim_b200 -- C ABI of the B200 (sm_100a) cone-beam projector library.
 *
 * Two families of entry points:
 *
 * 1. Drop-in replacements for the reference's CUDA MEX back ends.  Same argument
 *    order, types and array layouts; host pointers in, host pointers out;
 *    synchronous; return true on success (the reference returns bool, and its MEX
 *    gateway turns false into mexErrMsgTxt("Error: cbct_geom_mex() failed.")).
 *    Unlike the reference, errors never exit() the host process and inputs are
 *    never modified (the reference's CPU back-projectors scale the sinogram
 *    argument in place).
 *
 *      image   float[nz][ny][nx]        (MATLAB single [nx ny nz], x fastest)
 *      proj    float[noviews][nu][nv]   (MATLAB single [nv nu noviews], v fastest)
 *      map     bool[ny][nx]             (MATLAB logical [nx ny])
 *      betas   double[noviews] (radians), couchz float[noviews] (mm)
 *      detector_type: 1 flat panel, 0 curved (equiangular), 2 arc of radius ADD about the
 *      rotation axis (geom/cbct/cbct_proj3.c, cbct_back3.c: the distance-driven pair only;
 *      other methods return CTSIM_ERR_UNSUPPORTED)
 *
 *    Outputs are overwritten (the reference MEX allocates them zero-filled and
 *    accumulates; the result is the same).  Host buffers may be pageable (they are
 *    staged through the library's pinned buffers by a few host threads) or
 *    page-locked (copied directly); the results are identical.
 *
 * 2. Device-resident plans for callers that keep volumes and sinograms in GPU
 *    memory (FDK, OS-PWLS loops, batching).  A plan holds the per-view geometry
 *    tables and scratch buffers; its projector calls take device pointers and a
 *    CUDA stream (as void*), allocate nothing, and are asynchronous.
 *
 * Status codes returned by the plan API: see ctsim_status.
 */
#ifndef CTSIM_B200_H
#define CTSIM_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CTSIM_OK = 0,
    CTSIM_ERR_ARGUMENT = 1,    /* invalid sizes, null pointers, unknown method */
    CTSIM_ERR_CUDA = 2,        /* a CUDA runtime call or kernel launch failed */
    CTSIM_ERR_ALLOC = 3,       /* device or host allocation failed */
    CTSIM_ERR_UNSUPPORTED = 4, /* geometry outside what the kernels implement (a footprint wider than a
                                  kernel's row buffer, a non-DD method on the arc detector) */
    CTSIM_ERR_NO_DEVICE = 5    /* no usable sm_100 device */
} ctsim_status;

/* Projector methods (the reference's geom type strings). */
typedef enum {
    CTSIM_PROJ_DD = 0,  /* "proj,dd"  */
    CTSIM_PROJ_TF = 1,  /* "proj,tf"  */
    CTSIM_BACK_DD = 2,  /* "back,dd"  */
    CTSIM_BACK_TF = 3,  /* "back,tf"  */
    CTSIM_BACK_PD = 4,  /* "back,pd"  */
    CTSIM_BACK_HPD = 5, /* "back,hpd" */
    CTSIM_BACK_VAR = 6  /* "back,var": variance backprojection, geom/cbct/cbct_back_var.c:1 */
} ctsim_method;

/* OR'ed into CTSIM_BACK_DD / CTSIM_BACK_TF in ctsim_plan_backproject_ex and
 * ctsim_batch_backproject (no reference counterpart): the FP32 sinogram is already
 * multiplied by the plan's axial amplitude table, the per-pixel factor that A^T applies
 * first (geom/cbct/cbct_back.c:196-214), as ctsim_pwls_residual_scaled writes its
 * residual.  The backprojection then reads it as it is: no scaled copy, no scratch. */
#define CTSIM_INPUT_SCALED 0x100

/* Storage types of volumes and sinograms in the plan API (arithmetic is always FP32). */
typedef enum {
    CTSIM_F32 = 0,
    CTSIM_BF16 = 1,  /* __nv_bfloat16 */
    CTSIM_F16 = 2    /* __half */
} ctsim_dtype;

/* Last error message of the calling thread (never NULL). */
const char *ctsim_last_error(void);

/* Library version string. */
const char *ctsim_version(void);

/* ---------------------------------------------------------------------------
 * Family 1: drop-in host-pointer entry points.
 * ------------------------------------------------------------------------- */

/* Replaces cbct_proj_dd_gpu (geom/dd_cuda/cbct_dd_proj.c:407-432) and the CPU
 * cbct_proj_dd (geom/cbct/cbct_proj.c:217-242): distance-driven forward projection. */
bool ctsim_proj_dd(int nx, int ny, int nz, float dx, float dy, float dz, float offset_x, float offset_y,
                   float offset_z, int nu, int nv, float du, float dv, float offset_u, float offset_v, float sad,
                   float add, float sdd, int noviews, const double *betas, const float *couchz, int detector_type,
                   const float *image, float *proj, const bool *map);

/* Replaces cbct_back_dd_gpu (geom/dd_cuda/cbct_dd_back.c:299-324) and the CPU
 * cbct_back_dd (geom/cbct/cbct_back.c:136-161): matched distance-driven backprojection. */
bool ctsim_back_dd(int nx, int ny, int nz, float dx, float dy, float dz, float offset_x, float offset_y,
                   float offset_z, int nu, int nv, float du, float dv, float offset_u, float offset_v, float sad,
                   float add, float sdd, int noviews, const double *betas, const float *couchz, int detector_type,
                   float *image, const float *proj, const bool *map);

/* Replaces cbct_proj_tf_gpu (geom/sf_cuda/cbct_sf_proj.c:443) and the CPU cbct_proj_tf
 * (geom/cbct/cbct_proj.c:464-489): separable-footprint (trapezoid/rectangle) forward projection. */
bool ctsim_proj_tf(int nx, int ny, int nz, float dx, float dy, float dz, float offset_x, float offset_y,
                   float offset_z, int nu, int nv, float du, float dv, float offset_u, float offset_v, float sad,
                   float add, float sdd, int noviews, const double *betas, const float *couchz, int detector_type,
                   const float *image, float *proj, const bool *map);

/* Replaces cbct_back_tf_gpu (geom/sf_cuda/cbct_sf_back.c:334) and the CPU cbct_back_tf
 * (geom/cbct/cbct_back.c:375-400): matched separable-footprint backprojection. */
bool ctsim_back_tf(int nx, int ny, int nz, float dx, float dy, float dz, float offset_x, float offset_y,
                   float offset_z, int nu, int nv, float du, float dv, float offset_u, float offset_v, float sad,
                   float add, float sdd, int noviews, const double *betas, const float *couchz, int detector_type,
                   float *image, const float *proj, const bool *map);

/* Replaces cbct_back_pd_gpu (geom/fdk_cuda/cbct_back_pd.c:230-256) and the CPU cbct_back_pd
 * (geom/cbct/cbct_back.c:7-33): voxel-driven bilinear FDK backprojection.
 * offBoundary true = "back,pd" (rows off the detector dropped),
 * false = "back,hpd" (v clamped to [0.5, nv-1.5]). */
bool ctsim_back_pd(int nx, int ny, int nz, float dx, float dy, float dz, float offset_x, float offset_y,
                   float offset_z, int nu, int nv, float du, float dv, float offset_u, float offset_v, float sad,
                   float add, float sdd, int noviews, const double *betas, const float *couchz, int detector_type,
                   float *image, const float *proj, const bool *map, bool offBoundary);

/* String dispatch of the reference gateway (geom/cbct/cbct_geom_mex.c:253-312): type is one of
 * "proj,dd" "proj,tf" "back,dd" "back,tf" "back,pd" "back,hpd" "back,var"; data is the image for "proj,*"
 * and the sinogram for "back,*"; out is the sinogram or image. */
bool ctsim_cbct_geom(const char *type, int nx, int ny, int nz, float dx, float dy, float dz, float offset_x,
                     float offset_y, float offset_z, int nu, int nv, float du, float dv, float offset_u,
                     float offset_v, float sad, float add, float sdd, int noviews, const double *betas,
                     const float *couchz, int detector_type, const float *data, float *out, const bool *map);

/* The drop-in entry points above keep, per device, the last geometry's plan, device buffers
 * and streams between calls (same geometry scalars, betas, couchz and map: reused; anything
 * else: rebuilt).  They move the data in view chunks that overlap the kernels: the forward
 * projection goes back to the host chunk by chunk while later chunks compute, and the DD,
 * SF, pd/hpd and var backprojections take the sinogram in chunk by chunk while earlier chunks
 * are backprojected.  No reference counterpart (the reference MEX back ends allocate and
 * free per call and copy one view at a time).  Results do not depend on the cache or the
 * chunks, bit for bit. */
/* Frees the kept plan, buffers and streams now. */
ctsim_status ctsim_host_cache_release(void);
/* enabled = 0: free after every call, as the reference does; 1 (the default): keep. */
ctsim_status ctsim_host_cache_enable(int enabled);

/* ---------------------------------------------------------------------------
 * Family 2: device-resident plans.
 * ------------------------------------------------------------------------- */

typedef struct ctsim_plan ctsim_plan;

/* Geometry scalars in the reference's MEX order. */
typedef struct {
    int nx, ny, nz;
    float dx, dy, dz;
    float offset_x, offset_y, offset_z;
    int nu, nv;
    float du, dv;
    float offset_u, offset_v;
    float sad, add, sdd;
    int noviews;
    int detector_type;
} ctsim_geom;

/* Create a plan on the current CUDA device.  betas/couchz/map are HOST arrays
 * (map may be NULL = all columns on).  The plan allocates its view tables and
 * scratch once; projector calls on it allocate nothing. */
ctsim_status ctsim_plan_create(const ctsim_geom *geom, const double *betas, const float *couchz,
                               const bool *map, ctsim_plan **plan);
ctsim_status ctsim_plan_destroy(ctsim_plan *plan);

/* Stream-ordered plan (no reference counterpart; served reconstruction): its device
 * memory comes from a library-owned pool of the current device, allocated, uploaded
 * and -- at ctsim_plan_destroy, and ctsim_fdk_destroy for FDK objects built on it --
 * freed on `stream` without a device-wide synchronisation.  All work on the plan must
 * be ordered before its destruction on that stream, and the stream must outlive it. */
ctsim_status ctsim_plan_create_async(const ctsim_geom *geom, const double *betas, const float *couchz,
                                     const bool *map, void *stream, ctsim_plan **plan);

/* Return unused memory of the current device's library pool to the driver, keeping
 * at least keep_bytes. */
ctsim_status ctsim_pool_trim(size_t keep_bytes);

/* Launch shapes of a plan (no reference counterpart): the forward projector's
 * candidate-parallel thread groups (1, 2, 4, 8) and the 32-voxel z blocks per lane of
 * the A^T passes (back_mz for DD, back_mz_tf for SF) and of the FDK/var kernel (pd_mz),
 * each 1, 2, 4 or 8.  Plans start with a size rule; set_tuning changes the non-zero
 * fields (validated against the geometry).  The group count and the A^T z blocks change
 * the floating-point rounding of A and A^T (the summation order and the start of the
 * running row sums), never the footprints; the FDK/var z blocks change nothing. */
typedef struct {
    int proj_groups;
    int back_mz;
    int pd_mz;
    int back_mz_tf;
    int proj_rows;  /* row threads per forward group: a multiple of 32 up to ceil(nv/4) rounded
                       to whole warps; 32 makes each group one warp that walks only the rows
                       of each candidate's shadow */
    int proj_layout; /* column prefix sums: 1 plain sums, 2 (sum, slope) pairs (one 8-byte load
                        per evaluation; twice the bytes; plans whose pairs take at most 160 MB
                        start with 2 and may switch), 3 plain sums with each candidate column
                        copied into shared memory by the copy engine before its rows are summed */
    int proj_slots;  /* layout 3: prefix columns per stage buffer (two buffers), 1 .. 64 */
} ctsim_tuning;
ctsim_status ctsim_plan_get_tuning(const ctsim_plan *plan, ctsim_tuning *tuning);
ctsim_status ctsim_plan_set_tuning(ctsim_plan *plan, const ctsim_tuning *tuning);

/* Autotuner: times every valid launch shape of `method` on sample_views evenly spaced
 * views of the plan (<= 0: up to 64; the best shape depends on the grid, so pass the
 * view count of the real launches) (zero data, the plan's allocation mode for two temporary buffers),
 * keeps the fastest and records it for the shape class (method, volume and detector
 * sizes, detector type) so later plans of the class reuse it without timing.
 * Synchronises `stream`.  ctsim_autotune_clear forgets the recorded choices. */
ctsim_status ctsim_plan_autotune(ctsim_plan *plan, int method, int sample_views, void *stream, ctsim_tuning *chosen);
ctsim_status ctsim_autotune_clear(void);

/* Batched launches (no reference counterpart): the distance-driven or separable-footprint
 * A (CTSIM_PROJ_DD/TF) or A^T (CTSIM_BACK_DD/TF) of n plans -- different geometries, one
 * device -- with device buffers of any ctsim_dtype (per item; FP32 arithmetic, as the _ex
 * plan calls): `in` is the image (A) or the selected views' sinogram
 * (A^T), `out` the sinogram of the selected views or the image (overwritten; A^T times
 * scale).  After the per-plan pre-passes (column prefix sums, or the ampv pre-scaling)
 * the projector blocks of all plans run in ONE persistent grid per launch-shape class
 * (forward: row threads and candidate groups; backward: z blocks and row vectorisation),
 * at most 64 plans per grid.  Each plan's scratch is used, so a plan appears at most once
 * per call.  Results equal the per-plan calls bit for bit. */
typedef struct {
    ctsim_plan *plan;
    const void *in;
    void *out;
    int view_begin, view_stride, view_count;
    float scale;
    int in_dtype, out_dtype; /* ctsim_dtype of in and out (0: FP32); arithmetic is FP32 */
} ctsim_batch_item;
ctsim_status ctsim_batch_project(int method, const ctsim_batch_item *items, int n, void *stream);
ctsim_status ctsim_batch_backproject(int method, const ctsim_batch_item *items, int n, void *stream);

/* Bytes of device memory the plan holds (tables + scratch). */
size_t ctsim_plan_device_bytes(const ctsim_plan *plan);

/* Forward projection of views [view_begin, view_begin + view_count*view_stride) with
 * stride view_stride (ordered subsets: begin = isub % M, stride = M).  d_proj receives
 * view_count views, contiguous [view_count][nu][nv].  method: CTSIM_PROJ_DD / CTSIM_PROJ_TF. */
ctsim_status ctsim_plan_project(ctsim_plan *plan, int method, const float *d_image, float *d_proj,
                                int view_begin, int view_stride, int view_count, void *stream);

/* Backprojection of view_count views read contiguously from d_proj (same view selection
 * as ctsim_plan_project).  The image is overwritten with (scale * A^T y); map-off columns are 0.
 * method: CTSIM_BACK_DD / CTSIM_BACK_TF / CTSIM_BACK_PD / CTSIM_BACK_HPD / CTSIM_BACK_VAR. */
ctsim_status ctsim_plan_backproject(ctsim_plan *plan, int method, const float *d_proj, float *d_image,
                                    int view_begin, int view_stride, int view_count, float scale, void *stream);

/* The same with the storage type of the image and the sinogram given separately
 * (ctsim_dtype): BF16/FP16 inputs are widened to FP32 on load, every footprint sum
 * accumulates in FP32, outputs are rounded to their storage type on store. */
ctsim_status ctsim_plan_project_ex(ctsim_plan *plan, int method, const void *d_image, int image_dtype, void *d_proj,
                                   int proj_dtype, int view_begin, int view_stride, int view_count, void *stream);
ctsim_status ctsim_plan_backproject_ex(ctsim_plan *plan, int method, const void *d_proj, int proj_dtype,
                                       void *d_image, int image_dtype, int view_begin, int view_stride,
                                       int view_count, float scale, void *stream);

/* Synchronous: reports whether any kernel on this plan met a footprint larger than its
 * buffers, or a staged forward projection whose copy wait ran out (a device-side flag;
 * never expected for a valid plan).  Waits for the device, or for a stream-ordered plan
 * (ctsim_plan_create_async) for the plan's own stream only. */
ctsim_status ctsim_plan_check(ctsim_plan *plan);

/* ---------------------------------------------------------------------------
 * FDK reconstruction (fbp/reconFDK.m) on a plan.
 * ------------------------------------------------------------------------- */

typedef struct ctsim_fdk ctsim_fdk;

/* Replaces fbp/reconFDK.m:19-84 for one geometry: builds the cosine weights
 * (reconFDK.m:38-48), the ramp x window filter of fbp/filter/designFilter2.m (flat) or
 * designEquiangularFilter2.m (curved) with window "ram-lak" "shepp-logan" "cosine"
 * "hamming" "hann" "hann50|75|80" "B50|75|80" "C50|75|80" and crop, the Parker
 * short-scan weights (fbp/weights/shortScanParkerWeight.m) when short_scan != 0, and
 * dbeta (reconFDK.m:78-81).  Holds a filtered-sinogram scratch buffer. */
ctsim_status ctsim_fdk_create(ctsim_plan *plan, const char *window, float crop, int short_scan, ctsim_fdk **fdk);
ctsim_status ctsim_fdk_destroy(ctsim_fdk *fdk);

/* Weighted, ramp-filtered sinogram (reconFDK.m:51-76), device pointers, all views. */
ctsim_status ctsim_fdk_filter(ctsim_fdk *fdk, const float *d_sino, float *d_filtered, void *stream);

/* Full FDK: filter, back,hpd, times dbeta, times 10 (reconFDK.m:84).  Image overwritten. */
ctsim_status ctsim_fdk_run(ctsim_fdk *fdk, const float *d_sino, float *d_image, void *stream);

/* The same with the sinogram stored as sino_dtype (ctsim_dtype; widened to FP32 on load).
 * ctsim_fdk_run_ex keeps the filtered sinogram in sino_dtype too (FP32 filter arithmetic,
 * rounded once at its store; the backprojection reads it as it is), in a buffer of the
 * FDK object allocated at the first run of each size. */
ctsim_status ctsim_fdk_filter_ex(ctsim_fdk *fdk, const void *d_sino, int sino_dtype, float *d_filtered, void *stream);
ctsim_status ctsim_fdk_run_ex(ctsim_fdk *fdk, const void *d_sino, int sino_dtype, float *d_image, void *stream);

/* The dbeta the FDK scaling uses. */
float ctsim_fdk_dbeta(const ctsim_fdk *fdk);

/* Host-only: the frequency response H[order] of fbp/filter/designFilter2.m (detector_type 1)
 * or designEquiangularFilter2.m (0) for gamma = du, in double; order = max(64,
 * 2^nextpow2(2 nu - 1)) is returned in *order (H may be NULL to query it). */
ctsim_status ctsim_fdk_design_filter(int nu, float du, float sdd, int detector_type, const char *window, float crop,
                                     double *H, int *order);

/* ---------------------------------------------------------------------------
 * OS-PWLS building blocks (device pointers, asynchronous on stream).
 * ------------------------------------------------------------------------- */

/* statsrecon/pwls/computeWeightsPwls.m:8-9: w = (s - r)^2 / (s + v), w = 0 where s <= r. */
ctsim_status ctsim_pwls_weights(const float *d_counts, float r, float v, float *d_w, size_t n, void *stream);

/* Subset data term of statsrecon/pwls/reconPwlsSeSqs.m:57-74: d = ax - y, wd = w d, and
 * *d_phi += sum(w d^2) in FP64 (d_phi may be NULL). */
ctsim_status ctsim_pwls_residual(const float *d_ax, const float *d_y, const float *d_w, float *d_wd, size_t n,
                                 double *d_phi, void *stream);

/* The same with y and w stored as `dtype` (ctsim_dtype) and the weights stored divided by
 * w_scale (a power of two keeps FP16's range for photon-count weights); the residual is
 * formed in FP32. */
ctsim_status ctsim_pwls_residual_ex(const float *d_ax, const void *d_y, const void *d_w, int dtype, float w_scale,
                                    float *d_wd, size_t n, double *d_phi, void *stream);

/* ctsim_pwls_residual_ex for view_count views of `plan`'s detector, with the weighted
 * residual written already multiplied by the plan's axial amplitude table (wd = (w d) *
 * ampv per pixel, the product A^T forms first), for ctsim_plan_backproject_ex with
 * CTSIM_INPUT_SCALED; *d_phi accumulates sum(w d^2) as before (no reference counterpart:
 * it fuses the residual with the first step of the backprojection).  d_y may be NULL
 * (d = ax: the (w A1) * ampv of the SQS denominator).  d_wd may be d_ax. */
ctsim_status ctsim_pwls_residual_scaled(const ctsim_plan *plan, const float *d_ax, const void *d_y, const void *d_w,
                                        int dtype, float w_scale, float *d_wd, int view_count, double *d_phi,
                                        void *stream);

/* *d_acc += sum((a - b)^2) in FP64 (the iteration rmsd, reconPwlsSeSqs.m:81). */
ctsim_status ctsim_sqdiff(const float *d_a, const float *d_b, size_t n, double *d_acc, void *stream);

/* penalty/huberPenalty.m (kind 0, parameter delta) and penalty/quadPenalty.m (kind 1) in 3-D:
 * mode 0 adds the value to *d_value (FP64), mode 1 writes the gradient, mode 2 the curvature
 * into d_out ([nz][ny][nx]).  The quadratic gradient uses dQuad(d) = d (the reference's
 * dQuad has an empty body, penalty/quadPenalty.m:350-352). */
ctsim_status ctsim_penalty(int kind, int mode, float delta, int nx, int ny, int nz, const float *d_x, float *d_out,
                           double *d_value, void *stream);

/* One separable-quadratic-surrogate update (reconPwlsSeSqs.m:59-66):
 * x_new = x - (num + beta S(x)) / (precom + beta T(x)), negatives, NaN and Inf set to 0; the
 * penalty gradient S and curvature T are gathered inline; the denominator and step are
 * formed in FP64.  d_x and d_xnew must differ. */
ctsim_status ctsim_sqs_update(int kind, float beta, float delta, int nx, int ny, int nz, const float *d_x,
                              float *d_xnew, const float *d_num, const float *d_precom, void *stream);

/* One Nesterov subset step of statsrecon/pwls/reconPwlsSeNesterovSqs.m:65-87:
 * du = (num + beta S(z)) / (precom + beta T(x)) (FP64); x_new = z - du; s = s - t du (in
 * place); z_new = (1 - 1/t_next) x_new + (1/t_next) s, from the unclamped x_new and s; then
 * negatives, NaN and Inf of x_new, s and z_new set to 0.  t is the momentum of this step,
 * t_next = (1 + sqrt(1 + 4 t^2)) / 2 the one after it.  d_xnew and d_znew must differ from
 * d_z, d_x, d_s and from each other. */
ctsim_status ctsim_nesterov_update(int kind, float beta, float delta, int nx, int ny, int nz, const float *d_z,
                                   const float *d_x, float *d_s, const float *d_num, const float *d_precom,
                                   double t, double t_next, float *d_xnew, float *d_znew, void *stream);

/* ---------------------------------------------------------------------------
 * 2-D fan-beam distance-driven and separable-footprint pair (geom/fbct).
 * Image float[ny][nx] (MATLAB [nx ny]), sinogram float[noviews][nu] (MATLAB [nu noViews]).
 * ------------------------------------------------------------------------- */

/* Replaces fbct_geom_mex (geom/fbct/fbct_geom_mex.c:225-278) for type "proj,dd", "proj,tf",
 * "back,dd", "back,tf" (fbct_proj.c:153,292; fbct_back.c:80,225): host pointers, out
 * overwritten, synchronous; false (and ctsim_last_error) on any error. */
bool ctsim_fbct_geom(const char *type, int nx, int ny, float dx, float dy, float offset_x, float offset_y, int nu,
                     float du, float offset_u, float sad, float add, float sdd, int noviews, const double *betas,
                     int detector_type, const float *data, float *out);

typedef struct ctsim_fan_plan ctsim_fan_plan;
typedef struct {
    int nx, ny;
    float dx, dy, offset_x, offset_y;
    int nu;
    float du, offset_u;
    float sad, add, sdd;
    int noviews;
    int detector_type; /* 1 flat, 0 curved */
} ctsim_fan_geom;

/* Device plan of a fan-beam geometry (view table on the current device; betas on the host). */
ctsim_status ctsim_fan_plan_create(const ctsim_fan_geom *geom, const double *betas, ctsim_fan_plan **plan);
ctsim_status ctsim_fan_plan_destroy(ctsim_fan_plan *plan);
/* A (CTSIM_PROJ_DD / CTSIM_PROJ_TF) of views view_begin + k * view_stride, k < view_count, into
 * d_sino[view_count][nu] (overwritten). */
ctsim_status ctsim_fan_project(ctsim_fan_plan *plan, int method, const float *d_image, float *d_sino, int view_begin,
                               int view_stride, int view_count, void *stream);
/* scale * A^T (CTSIM_BACK_DD / CTSIM_BACK_TF) of d_sino[view_count][nu] into d_image (overwritten). */
ctsim_status ctsim_fan_backproject(ctsim_fan_plan *plan, int method, const float *d_sino, float *d_image,
                                   int view_begin, int view_stride, int view_count, float scale, void *stream);

/* ---------------------------------------------------------------------------
 * Sinogram pre-processing (the data step in front of the projectors).
 * ------------------------------------------------------------------------- */

/* sinogram/sim/simulateSimplePoissonData.m:161-190, monochromatic spectrum:
 * counts = Poisson(photons * exp(-line)) + sqrt(electronic_noise) * N(0, 1) per element, or,
 * with add_noise = 0, round(photons * exp(-line)).  photons = DQE * photonsTotal.  The draws
 * come from a Philox4x32-10 stream per element keyed by seed, so they depend only on
 * (seed, element index).  d_fallbacks (may be NULL) counts elements whose bounded
 * rejection loop gave up and returned round(lambda) (not expected in practice). */
ctsim_status ctsim_simulate_counts(const float *d_line, size_t n, float photons, float electronic_noise,
                                   uint64_t seed, int add_noise, float *d_counts, unsigned int *d_fallbacks,
                                   void *stream);

/* sinogram/log/computeSimplePoissonSinogramAttunation.m:14-54:
 * sino = -log(max(counts, 10) / source_intensity [./ flat]), d_flat (may be NULL) holding the
 * bowtie flat-field ratio of one view (nuv = nu * nv elements, sinogram layout). */
ctsim_status ctsim_log_attenuation(const float *d_counts, size_t n, float source_intensity, const float *d_flat,
                                   size_t nuv, float *d_sino, void *stream);

/* Matched distance-driven backprojection (same result as CTSIM_BACK_DD, within float
 * rounding) that allocates no device memory.  No counterpart in the reference: its MEX
 * back ends cudaMalloc and cudaFree on every call.
 *
 * For callers that must not allocate: a host framework that owns all device memory
 * through its own pool, a serving loop with a fixed memory budget, or code that cannot
 * afford the implicit device synchronisation of cudaMalloc/cudaFree.  d_proj
 * ([noviews][nu][nv]) and d_image ([nz][ny][nx], overwritten) are device pointers the
 * caller owns; betas, couchz and map (NULL = all columns on) are host arrays.
 *
 * Limit: the per-view table, the detector amplitude table and the map live in one
 * fixed 8 MiB array in device memory (each GPU that loads the library holds it until
 * the process exits); the call returns CTSIM_ERR_ARGUMENT when
 * noviews*44 + nu*nv*4 + nx*ny bytes (each part rounded up to 256) + 256 exceed it.
 * The first call on a device looks up that array's device address (set-up, once per
 * device); make that first call before any stream capture.  Every call rewrites the
 * shared array, so calls that overlap on the GPU (other streams, other host threads)
 * race; serialise them.  The work runs on `stream`, and the call returns when it has
 * finished: it reads back the kernel's row-buffer flag and returns CTSIM_ERR_UNSUPPORTED
 * if a column's detector rows did not fit (never for a geometry the size checks accept;
 * the image would be incomplete). */
ctsim_status ctsim_back_dd_noalloc(const ctsim_geom *geom, const double *betas, const float *couchz,
                                   const bool *map, const float *d_proj, float *d_image, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTSIM_B200_H */
