/*
 * shotsweep.h - C ABI of libshotsweep, the sm_100a (B200) implementation of
 * ShotSweep's physics hot path: the batched 2-D constant-density acoustic
 * finite-difference simulator and its exact discrete adjoint, which produce
 * surface gathers, per-shot velocity gradients, source illumination and
 * reverse-time-migration (RTM) images.
 *
 * The reference is pure Python (openfwi/physics/gpu.py); it has no FFI.  Each
 * entry point below replaces the computational core of one method of the
 * reference's `Sim` class or one module-level helper, and is what a ctypes
 * binding of that method calls (shotsweep_b200/_lib.py is that binding).
 *
 * Conventions
 *   - All array pointers are DEVICE pointers, C-contiguous float32 unless the
 *     name says f64.  Outputs are caller-allocated.
 *   - Every compute call is asynchronous and ordered on `stream` (a
 *     cudaStream_t passed as void*; NULL = legacy default stream).
 *   - Return value: SS_OK (0) or a negative ss_status; the message of the last
 *     failure on the calling thread is available from ss_last_error().
 *   - The simulation entry points need a device workspace of
 *     ss_workspace_bytes(...) bytes.  Device-side failures (a bounded wait that
 *     ran out) are recorded in the workspace; ss_workspace_status() reads them
 *     back after synchronising `stream`.
 *   - Per-solve geometry follows the reference: padded grid
 *     (nz+2*pad) x (nx+2*pad), sources and receivers on model row `src_row`,
 *     receivers at every model column, wavelet samples already scaled by the
 *     caller (the reference multiplies by 1e3, gpu.py:94).
 */
#ifndef SHOTSWEEP_H
#define SHOTSWEEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SS_MAX_SHOTS 16

typedef enum ss_status {
    SS_OK = 0,
    SS_ERR_INVALID = -1,      /* bad argument (shape, pointer, range)          */
    SS_ERR_UNSUPPORTED = -2,  /* geometry does not fit any kernel plan         */
    SS_ERR_CUDA = -3,         /* a CUDA runtime call failed                    */
    SS_ERR_TIMEOUT = -4,      /* a device-side bounded wait ran out            */
    SS_ERR_WORKSPACE = -5,    /* workspace missing or too small for one solve  */
    SS_ERR_NONFINITE = -6     /* observed gathers hold NaN or infinity         */
} ss_status;

/* Acquisition and grid of one batch (reference: openfwi/physics/constants.py:4-7,
 * Sim.__init__ gpu.py:77-96).  Defaults of the reference: nz=nx=70, nt=1000,
 * pad=40, n_shots=5, shot_cols={0,17,34,52,69}, src_row=1, dx=10, dt=1e-3,
 * r_coef=1e-5, vmax_damping=4500, amp_ref=2000. */
typedef struct ss_geometry {
    int32_t nz, nx;                     /* model cells (rows, columns)                    */
    int32_t nt;                         /* time steps                                     */
    int32_t pad;                        /* absorbing-layer width in cells (>= 2)          */
    int32_t n_shots;                    /* shots per velocity model (1..SS_MAX_SHOTS)     */
    int32_t src_row;                    /* model row of sources and receivers             */
    int32_t shot_cols[SS_MAX_SHOTS];    /* source columns in model coordinates            */
    double dx, dt;                      /* grid spacing (m) and time step (s)             */
    double r_coef;                      /* target reflection coefficient R of the layer   */
    double vmax_damping;                /* velocity in the damping constant (4500)        */
    double amp_ref;                     /* source-strength normalisation velocity (2000)  */
} ss_geometry;

typedef enum ss_mode {
    SS_MODE_FORWARD = 0,   /* gathers only                         */
    SS_MODE_GRADIENT = 1,  /* forward + adjoint -> gradient, illum  */
    SS_MODE_IMAGES = 2,    /* gradient + image epilogue             */
    SS_MODE_SEGMENT = 3    /* one checkpointed adjoint segment      */
} ss_mode;

/* Library version string. */
const char* ss_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* ss_last_error(void);

/* Bytes of device workspace that a call with this geometry, number of
 * velocity models and mode needs on the current device to keep every
 * co-resident cluster busy.  ss_gradient / ss_images accept a smaller
 * workspace and then keep fewer solves in flight (as many as it holds; at
 * least one).  Memory model of the reference: imaging_memory_bytes
 * (openfwi/physics/gpu.py:70-73). */
size_t ss_workspace_bytes(const ss_geometry* geom, int32_t n_models, int32_t mode);

/* Bytes of workspace for a call that keeps at most `slots` solves in flight
 * (per-solve scratch: the per-step history of one solve and its trace,
 * padded-gradient and gradient rows).  Needs no device: a caller with a
 * memory budget sizes its workspace with it before any launch.  Used by the
 * drop-in's imaging_memory_bytes (openfwi/physics/gpu.py:70-73). */
size_t ss_workspace_bytes_slots(const ss_geometry* geom, int32_t mode, int32_t slots);

/* The inverse: how many solves a workspace of `bytes` keeps in flight (0:
 * not even one; the plan's co-resident clusters cap it at launch).  Needs no
 * device. */
int32_t ss_workspace_slots(const ss_geometry* geom, int32_t mode, size_t bytes);

/* Reads the device-side status word of `workspace` after synchronising
 * `stream`: SS_OK, SS_ERR_TIMEOUT if a bounded wait ran out, or
 * SS_ERR_NONFINITE if the observed gathers held a non-finite sample (the
 * reference rejects those with ValueError, gpu.py:156-157; outputs of such a
 * call are undefined). */
int32_t ss_workspace_status(const void* workspace, void* stream);

/* Kernel plan for diagnostics: out[0..7] = cluster size (CTAs per solve),
 * threads per CTA, dynamic shared bytes per CTA, band rows per CTA, column
 * groups, rows per thread, co-resident clusters on this device, solves
 * in flight for n_models. */
int32_t ss_plan_info(const ss_geometry* geom, int32_t n_models, int32_t mode, int64_t out[8]);

/* Tile height (rows of its band each thread keeps in registers, 4 or 5) of
 * the plans of `mode` made after this call, process-wide; 0 restores the
 * default (5).  Taller tiles reuse more vertical neighbours from registers,
 * shorter ones allow more threads (warps) per CTA; a tuner times both and
 * sets the faster.  Every tile height computes the same values.  No
 * counterpart in the reference (its tensors have no tiles). */
int32_t ss_set_rows_per_thread(int32_t mode, int32_t rows);

/* Forward modelling.  Replaces Sim.forward / Sim.gathers (gpu.py:117-140).
 *   vel      [n_models, nz, nx]                    velocities (m/s)
 *   wavelet  [nt]                                  scaled source samples
 *   gathers  [n_models, n_shots, nt, nx]           output: receiver traces
 *   ckpt     NULL or [n_models, n_shots, ceil(nt/ckpt_interval), 2, nz+2pad, nx+2pad]
 *            output: wavefields (p0, p1) before every ckpt_interval-th step,
 *            as Sim.forward(store=True) keeps them (gpu.py:130-132); the
 *            caller zero-fills it (its 2-cell border is never written). */
int32_t ss_forward(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                   float* gathers, float* ckpt, int32_t ckpt_interval,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Per-shot gradient of 0.5*sum(w*(sim-obs)^2) and source illumination.
 * Replaces Sim._gradient / Sim.gradient (gpu.py:152-194).
 *   obs      [n_models, n_shots, nt, nx]   observed gathers
 *   v_mute   NULL (no mute) or [n_models]   mute velocities (gpu.py:142-150)
 *   grad     [n_models, n_shots, nz, nx]    output
 *   illum    [n_models, n_shots, nz, nx]    output: sum over steps of Laplacian^2 */
int32_t ss_gradient(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                    const float* obs, const float* v_mute, float t_mute,
                    float* grad, float* illum,
                    void* workspace, size_t workspace_bytes, void* stream);

/* RTM images: illumination-normalised negative gradients, optionally
 * Laplacian filtered.  Replaces Sim.images (gpu.py:196-210).
 *   img      [n_models, n_shots, nz, nx]    output
 *   illum    [n_models, n_shots, nz, nx]    output
 *   grad     NULL or [n_models, n_shots, nz, nx]  optional output */
int32_t ss_images(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                  const float* obs, const float* v_mute, float t_mute, float eps, int32_t laplacian,
                  float* img, float* illum, float* grad,
                  void* workspace, size_t workspace_bytes, void* stream);

/* Forward modelling and gradient with one source wavelet per velocity model.
 * The reference's multiscale FWI estimates a wavelet for each model and
 * frequency band (archive/toy/slopes/fwi.py:85-90, 144-146) and runs its
 * forward and gradient with it (fwi.py:46-77); these run a whole batch of
 * models, each with its own wavelet, in one launch.
 *   wavelets [n_models, nt]   scaled source samples of each model
 * Everything else as ss_forward (without checkpoints) and ss_gradient. */
int32_t ss_forward_wavelets(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelets,
                            float* gathers, void* workspace, size_t workspace_bytes, void* stream);
int32_t ss_gradient_wavelets(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelets,
                             const float* obs, const float* v_mute, float t_mute, float* grad, float* illum,
                             void* workspace, size_t workspace_bytes, void* stream);

/* Checkpointed adjoint for differentiation (torch.autograd): the forward
 * keeps only the states (p[t-1], p[t]) every K = ckpt_interval steps
 * (ss_forward with ckpt), and the gradient is rebuilt segment by segment,
 * last segment first.  Replaces the checkpoint/recompute loop of
 * Sim._gradient (gpu.py:169-184) with a given adjoint source instead of the
 * muted residual.  Per segment k (levels [kK, min((k+1)K, nt))):
 *   res        [n_models, n_shots, nt, nx]     adjoint source dJ/d(gathers)
 *   theta      [n_models, n_shots, 2, nz+2pad, nx+2pad]  scaled adjoint state,
 *              zero before the last segment, carried in place between calls
 *   gacc       [n_models, n_shots, nz+2pad, nx+2pad]     accumulator, zero at start
 *   illum_acc  [n_models, n_shots, nz, nx]               accumulator, zero at start
 *   src_acc    [n_models, n_shots]                       accumulator, zero at start
 * Workspace: ss_segment_workspace_bytes.  After segment 0, ss_gradient_finish
 * turns the accumulators into the per-shot gradient and illumination
 * (the fold and source term of gpu.py:185-187). */
size_t ss_segment_workspace_bytes(const ss_geometry* geom, int32_t n_models, int32_t ckpt_interval);
int32_t ss_adjoint_segment(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                           const float* ckpt, int32_t ckpt_interval, int32_t seg_index, const float* res,
                           float* theta, float* gacc, float* illum_acc, float* src_acc,
                           void* workspace, size_t workspace_bytes, void* stream);
int32_t ss_gradient_finish(const ss_geometry* geom, int32_t n_models, const float* vel, const float* gacc,
                           const float* src_acc, const float* illum_acc, float* grad, float* illum, void* stream);

/* Module helpers (gpu.py:33-67, 142-150, 105-107) on device arrays whose last
 * two axes are (n0, n1); `batch` is the product of the leading axes. */
int32_t ss_lap_f32(const float* p, float* out, int64_t batch, int32_t n0, int32_t n1, void* stream);
int32_t ss_lap_f64(const double* p, double* out, int64_t batch, int32_t n0, int32_t n1, void* stream);
int32_t ss_lap_adjoint_f32(const float* p, float* out, int64_t batch, int32_t n0, int32_t n1, void* stream);
int32_t ss_lap_adjoint_f64(const double* p, double* out, int64_t batch, int32_t n0, int32_t n1, void* stream);
/* g [batch, nz+2pad, nx+2pad] -> out [batch, nz, nx] (transpose of edge padding). */
int32_t ss_fold_edge_padding_f32(const float* g, float* out, int64_t batch, int32_t nz, int32_t nx,
                                 int32_t pad, void* stream);
int32_t ss_fold_edge_padding_f64(const double* g, double* out, int64_t batch, int32_t nz, int32_t nx,
                                 int32_t pad, void* stream);
/* Direct-wave mute weights [n_models, n_shots, nt, nx] (gpu.py:142-150). */
int32_t ss_mute_weights(const ss_geometry* geom, int32_t n_models, const float* v_mute, float t_mute,
                        float* out, void* stream);
/* Squared Courant numbers of the edge-padded model, c2 = v^2 (dt/dx)^2,
 * [n_models, nz+2pad, nx+2pad] (gpu.py:105-107). */
int32_t ss_c2_field(const ss_geometry* geom, int32_t n_models, const float* vel, float* out, void* stream);

/* RTM images without any device allocation: no counterpart in the
 * reference.  Some callers cannot call cudaMalloc when they need images: a
 * plugin host that hands over only input and output buffers, a framework
 * whose caching allocator owns all device memory, or a service that must not
 * allocate after start-up.  This entry point computes exactly what ss_images
 * computes (same arguments without the workspace), taking its scratch from a
 * fixed 32 MiB (33554432-byte) device array inside the library, which every
 * GPU that loads the library holds until the process exits.
 *   - Geometries whose single-solve scratch (per-step history, receiver
 *     traces, padded gradient) exceeds 32 MiB are rejected with
 *     SS_ERR_UNSUPPORTED; the 70x70 / 1000-step OpenFWI geometry needs about
 *     90 MB per solve and so needs ss_images.  Smaller problems run with as
 *     many solves in flight as fit in the array.
 *   - The call cannot be captured into a CUDA graph: it ends by waiting for
 *     its work (below), and returns SS_ERR_UNSUPPORTED when `stream` is
 *     capturing.
 *   - Every call shares the one array, and it keeps the previous call's
 *     contents: calls that overlap on the GPU (other streams, other host
 *     threads) race and corrupt each other's results.
 *   - The call waits for its work on `stream` and returns the device-side
 *     status (SS_ERR_NONFINITE, SS_ERR_TIMEOUT), since there is no workspace
 *     to read it from afterwards. */
int32_t ss_images_noalloc(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                          const float* obs, const float* v_mute, float t_mute, float eps, int32_t laplacian,
                          float* img, float* illum, float* grad, void* stream);

/* FP32 throughput probe (no counterpart in the reference: a diagnostic that
 * supplies the roofline denominator of the FP32 stencil kernels).  Launches
 * `blocks` x 256 threads, each running 8 independent FMA chains of `iters`
 * steps, scalar (packed = 0) or packed FP32x2 (packed = 1); *flops receives
 * the floating-point operations the launch performs (an FMA counts 2).  The
 * caller times the launch on `stream`; `out` must hold one float. */
int32_t ss_fp32_probe(float* out, int32_t blocks, int32_t iters, int32_t packed, double* flops, void* stream);

/* Failure-detection probe (no counterpart in the reference): one warp runs the
 * simulation kernels' bounded mbarrier wait on a barrier that nothing arrives
 * on; after limit_ms (0 < limit_ms <= 10000) it writes SS_ERR_TIMEOUT to
 * *status (device int) and returns, as a stalled solve would, without hanging
 * or faulting the GPU. */
int32_t ss_wait_probe(int32_t* status, double limit_ms, void* stream);

/* ---- Uneven batches ------------------------------------------------------
 * Models of different grid size, step count and shot count in one launch
 * sequence.  No counterpart in the reference, whose Sim is fixed to one
 * 70x70 grid, 1000 steps and 5 shots (gpu.py:59,95-96,103,126-128); each
 * solve computes exactly what ss_forward / ss_gradient / ss_images compute
 * for a batch holding only its own geometry.
 *
 * Solves are grouped into size classes: a class holds the solves whose
 * smallest fitting cluster (CTAs per solve) is the same, and runs as one
 * persistent launch whose clusters take solves longest-first.  `concurrent`
 * picks the streams: 0 runs the classes one after another on the caller's
 * stream (heaviest first); 1 alternates them between the caller's stream and
 * a second stream of the library, so that one class's tail overlaps the next
 * class's start; 2 puts the classes whose clusters leave many SMs idle (large
 * clusters pack the GPU's processing clusters badly) first on the caller's
 * stream and runs the others beside them on the second stream, filling those
 * SMs (falls back to 1 when the classes do not split).
 *
 * 1. ss_batch_plan (host): validates the items, forms the classes and the
 *    per-class launch shapes, and writes a self-contained plan of
 *    *plan_bytes bytes into `plan` (host memory; NULL: only report the
 *    sizes).  `cluster_by_class` (NULL, or SS_MAX_CLUSTER + 1 entries indexed
 *    by a class's smallest cluster at 5 rows per thread; an autotuner fills
 *    it) gives each size class its launch shape: bits 0-7 the cluster size
 *    (0 = that smallest cluster), bits 8-15 the tile height in rows per
 *    thread, 4..6 (0 = 5).  A solve that does not fit the chosen shape runs
 *    at the next cluster size that fits it.
 * 2. The caller copies the plan bytes unchanged to device memory.
 * 3. ss_batch_run (stream-ordered): runs every class; the same plan serves
 *    any number of runs with new data in the same layout. */
#define SS_MAX_CLUSTER 16

typedef struct ss_batch_item {          /* one velocity model (one background row) */
    int32_t nz, nx, nt, pad;
    int32_t n_shots, src_row;
    int32_t shot_cols[SS_MAX_SHOTS];
    int64_t vel_offset;   /* floats into vel: the model [nz][nx]                           */
    int64_t obs_offset;   /* floats into obs (gradient, images) or gathers (forward):
                             [n_shots][nt][nx]                                             */
    int64_t out_offset;   /* floats into img / illum / grad: [n_shots][nz][nx]             */
    float v_mute;         /* direct-wave mute velocity in m/s (gpu.py:142-150); <= 0: none */
    int32_t reserved;
} ss_batch_item;

typedef struct ss_physics {             /* shared by every item (constants.py, gpu.py:77-96) */
    double dx, dt, r_coef, vmax_damping, amp_ref;
} ss_physics;

typedef struct ss_batch_class_info {
    int32_t min_cluster;  /* the size class: smallest cluster fitting its solves */
    int32_t cluster;      /* CTAs per solve used                                 */
    int32_t n_solves;
    int32_t threads;      /* per CTA                                             */
    int32_t smem_bytes;   /* per CTA                                             */
    int32_t slots;        /* persistent clusters launched                        */
    int32_t stream;       /* 0: the caller's stream, 1: the library's second one */
    int32_t rows_per_thread;  /* tile height of the class's launch               */
    double cell_steps;    /* sum over its solves of padded cells x steps         */
} ss_batch_class_info;

int32_t ss_batch_plan(const ss_physics* phys, int32_t mode, const ss_batch_item* items, int32_t n_items,
                      const int32_t* cluster_by_class, int32_t concurrent, void* plan, size_t* plan_bytes,
                      size_t* workspace_bytes);
/* Smallest cluster (CTAs per solve) that fits the item in `mode`: its size
 * class; negative ss_status if none does. */
int32_t ss_batch_min_cluster(const ss_batch_item* item, int32_t mode);
/* The same at `rows` rows per thread (4..6): what an autotuner that picks a
 * class's tile height needs to know about each of its grids. */
int32_t ss_batch_min_cluster_rows(const ss_batch_item* item, int32_t mode, int32_t rows);
int32_t ss_batch_classes(const void* plan, ss_batch_class_info* out, int32_t max_classes, int32_t* n_classes);
/* wavelet: at least the batch's largest nt samples (scaled as for ss_forward).
 * gathers: forward mode output; img: images mode output; grad: gradient mode
 * output, optional in images mode; illum: gradient and images modes. */
int32_t ss_batch_run(const void* plan, const void* plan_device, const float* vel, const float* wavelet,
                     const float* obs, float t_mute, float eps, int32_t laplacian, float* gathers, float* img,
                     float* illum, float* grad, void* workspace, size_t workspace_bytes, void* stream);

/* ---- After the images: 2_process's cache epilogue, surface velocity and
 * training inputs (no FFI in the reference: these replace NumPy code that
 * 2_process.py and 3_train.py run on the host per model) ---- */

/* First-arrival surface velocity of one model's gathers
 * (background.py:19-83, estimate_surface_velocity): onsets at the first sample
 * whose |amplitude| exceeds frac x the trace's peak, line fits of the median
 * onset time per offset at 10-60 m, curvature, shot-to-shot spread and the
 * far-offset (120-250 m) refraction check.  status: SS_SURF_OK or the
 * reference's reason for raising ValueError. */
typedef enum ss_surface_status {
    SS_SURF_OK = 0,
    SS_SURF_NO_ONSETS = 1,    /* no nonzero onset traces                      */
    SS_SURF_FEW_NEAR = 2,     /* not exactly six distinct 10-60 m offsets      */
    SS_SURF_SLOPE = 3,        /* short-offset velocity outside 1400-4600 m/s   */
    SS_SURF_FEW_SHOTS = 4,    /* fewer than three shots with 4 near offsets    */
    SS_SURF_UNRELIABLE = 5,   /* RMSE > 2 ms, curvature or spread > 0.15       */
    SS_SURF_NONFINITE = 6     /* non-finite samples                           */
} ss_surface_status;

typedef struct ss_surface_estimate {
    double velocity;                 /* clip(1 / slope, 1500, 4500) m/s        */
    double confidence;
    double fit_rmse_ms;
    double short_offset_curvature;
    double shot_slope_spread;
    double far_offset_velocity;      /* NaN when the far slope is not positive */
    int32_t possible_refraction;
    int32_t status;                  /* ss_surface_status                      */
} ss_surface_estimate;

/* gathers [n_models][n_shots][nt][nx] f32 (device); src_x: HOST array of the
 * n_shots source positions in metres; out [n_models] (device). */
int32_t ss_surface_velocity(const float* gathers, int32_t n_models, int32_t n_shots, int32_t nt, int32_t nx,
                            const double* src_x, double dx, double dt, double frac, ss_surface_estimate* out,
                            void* stream);
/* Laterally constant backgrounds clip(v_surface[m] + rhos[k] trend[z], 1500, 4500)
 * (background.py:97-99) in float64, stored as f32 [n_models][n_rhos][nz][nx]. */
int32_t ss_backgrounds(const double* v_surface, const double* trend, const double* rhos, int32_t n_models,
                       int32_t n_rhos, int32_t nz, int32_t nx, float* out, void* stream);
/* The image cache of 2_process.py:206-210: per model, rows [0, zero_rows) of
 * every image zeroed, scale = the q-th percentile of |img| over the model's
 * n_images x nz x nx values (NumPy's linear interpolation on float32 data),
 * out = binary16(clip(img / scale, -clip, clip)).  img and out
 * [n_models][n_images][nz][nx]; scale [n_models] f32; status [n_models]:
 * SS_OK, SS_ERR_NONFINITE or SS_ERR_INVALID (scale <= 0), which 2_process
 * turns into ValueError. */
int32_t ss_image_cache(const float* img, int32_t n_models, int32_t n_images, int32_t nz, int32_t nx,
                       int32_t zero_rows, double q, float clip, uint16_t* out, float* scale, int32_t* status,
                       void* stream);
/* Training inputs: the stored form binary16(sign(g) log1p(|g|)) (3_train.py:157),
 * and a batch's float32 copy of it divided by the normalisation scale (3_train.py:198). */
int32_t ss_signed_log1p_f16(const float* g, int64_t n, uint16_t* out, void* stream);
int32_t ss_f16_scaled(const uint16_t* in, int64_t n, float scale, float* out, void* stream);
/* Training targets (3_train.py:158,188-189): y = (vel - 3000) / 1500 over n values, and
 * when vref is given, vref [n_models][nz][nx] = clip((v_surface[m] + trend[z] - 3000) / 1500, -1, 1). */
int32_t ss_velocity_targets(const float* vel, int64_t n, float* y, const float* v_surface, const float* trend,
                            int32_t n_models, int32_t nz, int32_t nx, float* vref, void* stream);

/* ---- Learned velocity proposal: tensor-core kernels (no counterpart in the
 * reference's physics; its networks are PyTorch modules, 3_train.py:219-260) ---- */

/* C[M][N] = A[M][K] . B[N][K]^T on the tcgen05 tensor cores: A and B BF16,
 * row-major with K innermost (row strides lda, ldb in elements, multiples of
 * 8, 16-byte aligned bases), F32 accumulation in tensor memory.  Epilogues:
 *   SS_EPI_F32             C (float) = acc
 *   SS_EPI_F32_ADD         C (float) += acc (atomic; the K loop may be split
 *                          over `splits` CTAs, 0 = chosen to fill the GPU)
 *   SS_EPI_BIAS_LRELU_BF16 C (BF16) = leaky_relu(acc + bias[n], slope)
 *   SS_EPI_BIAS_F32        C (float) = acc + bias[n] (bias may be NULL)
 * err: device int, set non-zero if a bounded wait of the pipeline ran out. */
typedef enum ss_gemm_epilogue {
    SS_EPI_F32 = 0,
    SS_EPI_F32_ADD = 1,
    SS_EPI_BIAS_LRELU_BF16 = 2,
    SS_EPI_BIAS_F32 = 3
} ss_gemm_epilogue;
int32_t ss_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                     int32_t epi, void* C, int64_t ldc, const float* bias, float slope, int32_t splits,
                     int32_t* err, void* stream);
/* ss_gemm_bf16 with operands stored either way: `layout` bit 0 set means A is
 * stored K-outer (A[k][m] at A + k*lda + m, lda >= M), bit 1 the same for B
 * (B[k][n] at B + k*ldb + n, ldb >= N).  The tensor cores read such operands
 * in place through M/N-major shared-memory descriptors, so C = A^T B^T-style
 * products (a weight gradient from the activations as they are stored) need
 * no transpose pass.  Layouts 0, 2 and 3; M/N-major strides obey the same
 * multiple-of-8 and alignment rules. */
int32_t ss_gemm_bf16_layout(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N,
                            int32_t K, int32_t layout, int32_t epi, void* C, int64_t ldc, const float* bias,
                            float slope, int32_t splits, int32_t* err, void* stream);

/* Convolution plumbing (NHWC BF16 activations).  conv[11] = {B, Hin, Win, Cin,
 * KH, KW, stride_h, stride_w, pad_h, pad_w, up}: the input is read through a
 * nearest-neighbour upsampling by `up`; Hout = (Hin*up + 2 pad_h - KH) / stride_h + 1
 * (likewise W); column index k = (kh*KW + kw)*Cin + c.
 *   ss_im2col_bf16        cols [pixels][Kc] (k >= KH*KW*Cin zero)
 *   ss_col2im16_lrelu_bf16 dpre[pixel][c] (row stride ldp) = leaky_relu'(y) x
 *                         the sum of the BF16 column gradients dcols
 *                         [pixels_out][Kc] that read input element (pixel, c);
 *                         y: the input map (Cin % 8 == 0 with Cin / 8 a power
 *                         of two, Kc % 8 == 0, 16-byte aligned dcols and y; at
 *                         most 2^31 - 1 input elements / 8)
 *   ss_bias_grad_bf16     db[c] += sum over rows of dpre[row][c]
 * Output head: crop [off, off+n)^2 of x [B][H][W][C], 3x3 convolution with
 * zero padding, bias, tanh; head[6] = {B, H, W, C, off, n}; weights w[9][C].
 *   ss_head_backward      dw += .., db += .., and dpre_x [B][H][W][C] =
 *                         leaky_relu'(x) x the input gradient (zero outside the crop)
 * ss_l1_tanh_loss         loss_sum += sum |pred - target|, dpre = sign(pred - target)/n x (1 - pred^2)
 * ss_adamw                one AdamW step on float parameters (optional BF16 copy); the learning
 *                         rate and the step counter (incremented first) are device values
 * ss_gather_rows_f32      out[b][:] = src[ids[b]][:] (rows of `row` floats)
 * ss_gathers_nhwc_bf16    network input: stored float16 gathers [n][S][T][X] of
 *                         samples ids[0..B) as BF16 [B][T][X][S] / scale (3_train.py:198) */
int32_t ss_im2col_bf16(const void* x, const int32_t* conv, int32_t Kc, void* cols, void* stream);
int32_t ss_col2im16_lrelu_bf16(const void* dcols, const int32_t* conv, int32_t Kc, const void* y, float slope,
                               void* dpre, int64_t ldp, void* stream);
int32_t ss_bias_grad_bf16(const void* dpre, int64_t ld, int64_t M, int32_t C, float* db, void* stream);
int32_t ss_head_forward(const void* x, const int32_t* head, const float* w, const float* bias, float* out, void* stream);
int32_t ss_head_backward(const void* x, const int32_t* head, const float* w, const float* dpre, float slope, float* dw,
                         float* db, void* dpre_x, void* stream);
int32_t ss_l1_tanh_loss(const float* pred, const float* target, int64_t n, float* loss_sum, float* dpre, void* stream);
int32_t ss_adamw(float* p, const float* grad, float* m, float* v, int64_t n, const float* lr, float b1, float b2,
                 float eps, float wd, int32_t* step, void* p_bf16, void* stream);
int32_t ss_gather_rows_f32(const float* src, const int32_t* ids, int32_t B, int64_t row, float* out, void* stream);
int32_t ss_gathers_nhwc_bf16(const uint16_t* stored, const int32_t* ids, int32_t B, int32_t S, int32_t T, int32_t X,
                             float scale, void* out, void* stream);

/* ---- L-BFGS full-waveform inversion, batched over models (the reference's
 * archive/toy/slopes/fwi.py:130-164 for many models at once; one CTA per model) ----
 * ss_fwi_precondition  out[m] = mute * smooth_x(smooth_z(mute * sum_s grads[m][s]))
 *                      (fwi.py:142-143; Gaussian of sigma `smooth` cells, radius
 *                      int(3 sigma) + 1, edge padding, slopes.py:20-26)
 * ss_fwi_misfit        J[m] = 0.5 sum (sim - obs)^2 over per_model values (float64)
 * ss_lbfgs_direction   d[m] from g[m] and the model's last count[m] (s, y) pairs
 *                      (slots next[m]-count[m] .. next[m]-1 of S, Y [B][mem][n]);
 *                      first step scaled to max |d| = cap, steepest descent of
 *                      max |d| = cap (and count[m] = 0) when g.d >= 0; gd[m] = g.d
 * ss_fwi_trial         vt[m] = clip(v[m] + step[m] d[m], lo, hi) where mask[m]
 * ss_lbfgs_push        where accept[m]: push (vt - v, gn - g) if s.y > 1e-12, then
 *                      v = vt, g = gn */
int32_t ss_fwi_precondition(const float* grads, int32_t B, int32_t S, int32_t nz, int32_t nx, float smooth, float* out,
                            void* stream);
int32_t ss_fwi_misfit(const float* sim, const float* obs, int32_t B, int64_t per_model, double* J, void* stream);
int32_t ss_lbfgs_direction(const float* g, const float* S, const float* Y, int32_t* count, const int32_t* next,
                           const int32_t* active, int32_t B, int32_t n, int32_t mem, float cap, float* d, double* gd,
                           void* stream);
int32_t ss_fwi_trial(const float* v, const float* d, const float* step, const int32_t* mask, int32_t B, int32_t n,
                     float lo, float hi, float* vt, void* stream);
int32_t ss_lbfgs_push(float* v, const float* vt, float* g, const float* gn, float* S, float* Y, int32_t* count,
                      int32_t* next, const int32_t* accept, int32_t B, int32_t n, int32_t mem, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SHOTSWEEP_H */
