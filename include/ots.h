/*
 * ots.h -- C ABI of the overlapped time-tiling stencil engine (libots.so).
 *
 * One B200, FP32, thirteen stencils.  The entry points take the parameter
 * surface of the reference's kernel-generator-plus-runner programs
 * (jholewinski/ics-12-overlapped-tiling, opencl/<stencil>/<stencil>.cpp) and
 * replace, in one library, what each runner did by hand:
 *
 *   reference                                         here
 *   ---------------------------------------------    ------------------------
 *   GeneratorParams + computeDerived()                ots_plan_create,
 *     (opencl/jacobi-2d/jacobi-2d.cpp:21-127)           ots_plan_geometry
 *   XGenerator::generate() -> OpenCL source,          compiled sm_100a kernels
 *     cl::Program::build                                chosen by ots_plan_create
 *     (opencl/jacobi-2d/jacobi-2d.cpp:162-173,741-780)
 *   hostData fill + enqueueWriteBuffer x2             ots_fill_reference,
 *     (opencl/jacobi-2d/jacobi-2d.cpp:787-802,874-886)  ots_upload
 *   launch loop, swap(in,out), events, rtclock        ots_run
 *     (opencl/jacobi-2d/jacobi-2d.cpp:899-948)
 *   enqueueReadBuffer(*inputBuffer)                   ots_download
 *     (opencl/jacobi-2d/jacobi-2d.cpp:952-954)
 *   printProgramParameters + printValue keys          ots_describe
 *     (opencl/common/inc/ProgramGenerator.hpp:19-66)
 *   CLContext (opencl/common/src/CLContext.cpp:11-45) ots_device_info
 *   throwOnError (CLContext.cpp:50-56), "ERROR: ..."  ots_status +
 *     (opencl/jacobi-2d/jacobi-2d.cpp:682-690)          ots_last_error
 *
 * Host arrays use the reference layout: P^d floats per field, x fastest,
 * P = ots_geometry.padded_size, interior cells at [padding, padding+real_size)
 * on every axis, every other cell zero (zero Dirichlet ring).  Device arrays
 * are plan-owned.  No call throws; every call returns an ots_status and
 * records a message for ots_last_error() (per thread).
 *
 * Threading: a plan is used by one host thread at a time; distinct plans may
 * be used concurrently from distinct threads.
 */
#ifndef OTS_H
#define OTS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ots_status {
  OTS_OK = 0,
  OTS_ERR_INVALID_ARGUMENT = 1,
  OTS_ERR_INVALID_GEOMETRY = 2, /* reference: "Consistency error!" / assert */
  OTS_ERR_SMEM_TOO_LARGE = 3,   /* reference: "Not enough local memory ..." */
  OTS_ERR_BLOCK_TOO_LARGE = 4,  /* reference: "Block dimensions are too large!" */
  OTS_ERR_CUDA = 5,
  OTS_ERR_TIMEOUT = 6,          /* a bounded device wait gave up */
  OTS_ERR_UNSUPPORTED = 7,
  OTS_ERR_NO_DEVICE = 8,
  OTS_ERR_OUT_OF_MEMORY = 9
} ots_status;

/* Stencil ids; names as the reference runners (opencl/<name>/). */
typedef enum ots_stencil {
  OTS_JACOBI_1D = 0,
  OTS_JACOBI_1D_5PT = 1,
  OTS_JACOBI_1D_7PT = 2,
  OTS_JACOBI_2D = 3,
  OTS_JACOBI_3D = 4,
  OTS_POISSON_2D = 5,
  OTS_POISSON_3D = 6,
  OTS_GRADIENT_2D = 7,
  OTS_GRADIENT_3D = 8,
  OTS_FDTD_2D = 9,
  OTS_RICIAN_DENOISE_2D = 10,
  OTS_CDSC_TV_UPDATE_2D = 11,
  OTS_CS_3D = 12,
  OTS_NUM_STENCILS = 13
} ots_stencil;

/* Geometry derivation.  COMPAT truncates the problem to a multiple of the
 * reference's sizeLCM and puts E on y in 3D, exactly as computeDerived does;
 * NATIVE keeps the exact problem size (partial edge tiles) and puts E on z
 * in 3D. */
typedef enum ots_engine { OTS_ENGINE_NATIVE = 0, OTS_ENGINE_COMPAT = 1 } ots_engine;

/* Kernel family.  TILE: overlapped time tile in every dimension (the
 * reference scheme).  STREAM: overlapped in x/y, streamed along z with all T
 * time levels in flight (3D star stencils).  PLAIN: one time step per launch
 * (the comparator).  TEX: the TILE scheme with the first-step loads through
 * the texture unit (opencl/jacobi-2d-tex/jacobi-2d-tex.cpp; 2D single-field
 * stencils, E <= 8).  AUTO picks STREAM where available in 3D, else TILE. */
typedef enum ots_kernel {
  OTS_KERNEL_AUTO = 0,
  OTS_KERNEL_TILE = 1,
  OTS_KERNEL_STREAM = 2,
  OTS_KERNEL_PLAIN = 3,
  OTS_KERNEL_TEX = 4
} ots_kernel;

/* Arithmetic variant where the reference and the benchmark definition
 * differ.  OTS_VARIANT_BASELINE: jacobi-3d weight 1/7; Poisson as a Jacobi sweep with RHS
 * f and h^2 (5-/7-point); FDTD with the standard Hz sign and the Ey row-0
 * source.  OTS_VARIANT_REF: the reference kernels' arithmetic (0.143f; 8c-sum8 and
 * 26c-sum26; +Ey in the Hz update, no source).  OTS_VARIANT_FAST (rician-denoise-2d,
 * cdsc-tv-update-2d, cs-3d only): the baseline arithmetic with every division
 * replaced by the approximate PTX division (div.approx.ftz.f32, 2 ulp;
 * subnormals flushed) and cs-3d's 1/sqrt terms in float rsqrt -- the latitude the reference's OpenCL build gave its
 * kernels (default options, single-precision '/' within 2.5 ulp;
 * opencl/rician-denoise-2d/rician-denoise-2d.cpp:662); results are no longer
 * bit-reproducible against an IEEE CPU loop, only within the tolerance the
 * tests state. */
typedef enum ots_variant {
  OTS_VARIANT_BASELINE = 0,
  OTS_VARIANT_REF = 1,
  OTS_VARIANT_FAST = 2
} ots_variant;

typedef struct ots_params {
  int32_t stencil;             /* ots_stencil */
  int32_t problem_size;        /* -n/--problem-size */
  int32_t time_steps;          /* -t/--time-steps */
  int32_t time_tile;           /* -s/--time-tile-size (T) */
  int32_t block_x;             /* -x/--block-size-x (threads) */
  int32_t block_y;             /* -y/--block-size-y */
  int32_t block_z;             /* -z/--block-size-z */
  int32_t elements_per_thread; /* -e/--elements-per-thread (E) */
  int32_t engine;              /* ots_engine */
  int32_t kernel;              /* ots_kernel */
  int32_t variant;             /* ots_variant */
  int32_t phase_limit;         /* -p/--phase-limit: 0 full, 1/2/3 partial kernels */
  float coef;                  /* averaging weight; 0 = the stencil's default */
  float h2;                    /* Poisson h^2; 0 = 1/(real_size-1)^2 */
  int32_t device;              /* CUDA device ordinal */
  int32_t cluster_y;           /* stream kernel: CTAs per thread-block cluster
                                  stacked along y (1..8; 0 or 1 = none).  The
                                  cluster shares one tile of cluster_y * block_y
                                  * E rows, so the 2T-row y halo is recomputed
                                  once per cluster instead of once per CTA. */
  int32_t stream_impl;         /* stream kernel arithmetic: 0 = the packed-FP32
                                  kernels where they apply -- 3D: jacobi-3d and
                                  poisson-3d, T <= 4, no clusters, n a multiple
                                  of 4, the block shapes 16x16, 16x8, 8x16 at
                                  E = 4 and 16x32, 32x16, 16x16 at E = 2; 2D:
                                  jacobi-2d and poisson-2d (baseline) -- else
                                  the scalar ones; 1 = always the scalar
                                  kernels.  Both give identical bits. */
  int32_t reserved[5];         /* must be zero */
} ots_params;

/* Derived values: the reference's GeneratorParams fields plus what the
 * chosen kernel actually launches. */
typedef struct ots_geometry {
  int32_t dims;
  int32_t radius;              /* true per-step dependence radius */
  int32_t num_fields;          /* evolving fields (ping-ponged) */
  int32_t num_aux;             /* read-only fields */
  int32_t padding;             /* host-layout ring width */
  int32_t padded_size;         /* host-layout P */
  int32_t real_size;           /* interior cells per axis */
  int32_t size_lcm;
  int32_t comps[3];            /* cells computed per CTA (incl. halo) */
  int32_t real_per_block[3];   /* interior cells written per CTA */
  int32_t num_blocks[3];       /* grid */
  int32_t shared_size[3];      /* reference sharedSize{X,Y,Z} */
  int32_t threads[3];          /* CTA shape launched */
  int32_t kernel;              /* resolved ots_kernel */
  int32_t e_axis;              /* axis E multiplies: 0 x, 1 y, 2 z */
  int32_t launches;            /* ceil(time_steps / T) */
  int32_t registers;           /* per thread, from cudaFuncGetAttributes */
  int64_t shared_bytes;        /* dynamic shared memory per CTA */
  int64_t interior_points;     /* real_size^dims */
  double flops_per_point;      /* the reference's per-point constant */
  double useful_ratio;         /* reference "Useful Ratio" */
  float coef;                  /* averaging weight in effect */
  float h2;                    /* Poisson h^2 in effect */
  int32_t ctas_per_sm;         /* resident CTAs per SM of the chosen kernel */
  int32_t sm_count;            /* SMs of the device */
} ots_geometry;

typedef struct ots_timing {
  double event_ms;             /* cudaEvent: first launch start -> last end */
  double wall_s;               /* host wall clock around launch + sync */
  int32_t launches;
  int32_t steps;
} ots_timing;

typedef struct ots_plan ots_plan;

/* ---- errors / device ------------------------------------------------- */

/* Message of the last failing call on this thread ("" if none). */
const char* ots_last_error(void);
const char* ots_status_string(ots_status s);

/* Device name, SM count, shared memory per block (opt-in), global memory. */
ots_status ots_device_info(int32_t device, char* name, size_t name_len, int32_t* sm_count,
                           int64_t* smem_per_block, int64_t* global_mem);

/* ---- stencil metadata -------------------------------------------------- */

const char* ots_stencil_name(int32_t stencil);
int32_t ots_stencil_from_name(const char* name); /* -1 if unknown */
int32_t ots_stencil_dims(int32_t stencil);
int32_t ots_stencil_num_fields(int32_t stencil);
int32_t ots_stencil_num_aux(int32_t stencil);
/* The performance-model constants the reference runner prints for this
 * stencil (opencl/jacobi-2d/jacobi-2d.cpp:1029-1036 and the matching lines of
 * each runner), in the order phase2_global_loads, phase2_shared_loads,
 * compute_per_point, phase3_shared_loads, phase4_global_stores,
 * shared_stores, num_fields, data_size.  OTS_ERR_UNSUPPORTED for the runners
 * that print none (jacobi-1d-5pt, jacobi-1d-7pt, cs-3d).  Needs no GPU. */
ots_status ots_stencil_model_constants(int32_t stencil, double out[8]);

/* Fill P^d host arrays (state fields then aux fields, as the reference
 * interleaves them per cell) with srand(seed); rand()/(RAND_MAX+1.0f) over
 * the interior, zero on the ring (opencl/poisson-2d/poisson-2d.cpp:611-621). */
ots_status ots_fill_reference(int32_t dims, int32_t padded_size, int32_t padding,
                              int32_t real_size, uint32_t seed, float* const* fields,
                              int32_t num_fields);

/* The image the Rician and TV workloads start from (no counterpart in the
 * reference, whose fill for these runners is disabled,
 * opencl/rician-denoise-2d/rician-denoise-2d.cpp:694-708): `count` disks of
 * constant intensity (uniform [0.2, 1.0)), radius uniform [n/64, n/12),
 * centres uniform over the grid, drawn in order over `background`; then
 * Rician noise f = sqrt((s + n1)^2 + n2^2), n1, n2 ~ N(0, sigma^2).  Seeded
 * (SplitMix64 uniforms, Box-Muller normals).  noisy (and clean, if not NULL):
 * n x n floats, row-major.  Needs no GPU. */
ots_status ots_fill_disks(int32_t n, uint64_t seed, int32_t count, float background, float sigma,
                          float* noisy, float* clean);

/* ---- plans -------------------------------------------------------------- */

/* Derive the geometry, pick and validate the kernel instantiation, allocate
 * device buffers.  Replaces GeneratorParams::computeDerived + generate() +
 * program build (opencl/jacobi-2d/jacobi-2d.cpp:84-126, 162-173, 741-780). */
ots_status ots_plan_create(const ots_params* params, ots_plan** out);
void ots_plan_destroy(ots_plan* plan);
ots_status ots_plan_geometry(const ots_plan* plan, ots_geometry* out);

/* Derive the geometry without allocating (what the reference prints before
 * running).  With a CUDA device visible this also resolves and validates the
 * kernel exactly as ots_plan_create does (registers, shared bytes, resident
 * CTAs per SM); without one it is the reference derivation only. */
ots_status ots_derive_geometry(const ots_params* params, ots_geometry* out);

/* Copy host fields (reference layout, P^d each) into the plan.  `state` has
 * num_fields arrays, `aux` num_aux arrays (may be NULL when num_aux == 0).
 * Replaces the two enqueueWriteBuffer calls (jacobi-2d.cpp:874-886). */
ots_status ots_upload(ots_plan* plan, const float* const* state, const float* const* aux);

/* Same, from dense interior arrays (real_size^dims floats, no ring). */
ots_status ots_upload_interior(ots_plan* plan, const float* const* state,
                               const float* const* aux);

/* Run time_steps steps: ceil(S/T) launches ping-ponging the state buffers
 * (jacobi-2d.cpp:905-931).  `kernel` overrides the plan's kernel family for
 * this run (OTS_KERNEL_AUTO keeps it).  The state advances in place, so a
 * second call continues from the first call's result.  `timing` may be NULL. */
ots_status ots_run(ots_plan* plan, int32_t kernel, ots_timing* timing);

/* Enqueue the run on the plan's stream and return without synchronising
 * (for CUDA-graph capture and timed loops); ots_sync waits for it. */
ots_status ots_run_async(ots_plan* plan, int32_t kernel);
ots_status ots_sync(ots_plan* plan);

/* Copy the current state back (reference layout / dense interior);
 * replaces enqueueReadBuffer(*inputBuffer) (jacobi-2d.cpp:952-954). */
ots_status ots_download(ots_plan* plan, float* const* state);
ots_status ots_download_interior(ots_plan* plan, float* const* state);

/* The four copies above, enqueued on the plan's stream without waiting
 * (the reference's non-blocking enqueueWriteBuffer/enqueueReadBuffer,
 * jacobi-2d.cpp:874-886, 952-954, with blocking off).  Host arrays must stay
 * valid and unchanged until ots_sync returns; with page-locked host memory
 * (ots_host_register) the copies overlap other plans' kernels, so several
 * plans on one GPU can pipeline upload, run and download of independent
 * problems. */
ots_status ots_upload_async(ots_plan* plan, const float* const* state, const float* const* aux);
ots_status ots_upload_interior_async(ots_plan* plan, const float* const* state,
                                     const float* const* aux);
ots_status ots_download_async(ots_plan* plan, float* const* state);
ots_status ots_download_interior_async(ots_plan* plan, float* const* state);

/* Report the reference runner's key/value lines (printProgramParameters and
 * the per-stencil model constants, jacobi-2d.cpp:1029-1037) through `kv`. */
typedef void (*ots_kv_fn)(const char* key, const char* value, void* user);
ots_status ots_describe(const ots_plan* plan, ots_kv_fn kv, void* user);

/* Device pointers of the plan's current state / aux buffers (dense interior
 * layout, x fastest), and its stream, for callers that keep data on the
 * GPU between runs. */
ots_status ots_plan_device_state(const ots_plan* plan, int32_t field, float** device_ptr);
ots_status ots_plan_device_aux(const ots_plan* plan, int32_t field, float** device_ptr);
ots_status ots_plan_stream(const ots_plan* plan, void** cuda_stream);

/* -c/--dump-clocks (opencl/jacobi-2d/jacobi-2d.cpp:178-204, :484-508,
 * :957-996): with recording on, every tile-kernel launch stores per warp the
 * SM id and %clock at five points -- entry, after set-up, after the global
 * load and first step, after the in-tile steps, after the write-back -- and
 * the last launch's records stay.  ots_plan_clock_records copies up to
 * `capacity` of them (block-major, warps in order) and sets *count to the
 * number available (0 if the last run was not the tile kernel). */
typedef struct ots_clock_record {
  uint32_t block_x, block_y, block_z, warp, sm;
  uint32_t clock[5];
} ots_clock_record;
ots_status ots_plan_enable_clocks(ots_plan* plan, int32_t enable);
ots_status ots_plan_clock_records(ots_plan* plan, ots_clock_record* out, int64_t capacity,
                                  int64_t* count);

/* Limit of every bounded device wait of the plan's 3D stream kernel (its
 * TMA ring barriers), 2 s by default; a wait that runs out makes the run
 * return OTS_ERR_TIMEOUT and leaves the context usable.  No reference
 * counterpart (the reference's in-order OpenCL queue has no device waits). */
ots_status ots_plan_set_wait_limit(ots_plan* plan, double seconds);
/* Test hook, no reference counterpart: with plane >= 0 the first CTA of the
 * 3D stream kernel arms the ring barrier of that running plane but never
 * loads it, so its wait runs out (OTS_ERR_TIMEOUT); -1 turns it off. */
ots_status ots_plan_debug_hold_plane(ots_plan* plan, int32_t plane);

/* Page-lock a caller's host buffer so uploads/downloads run as async DMA. */
ots_status ots_host_register(void* ptr, size_t bytes);
ots_status ots_host_unregister(void* ptr);

/* ---- batched grids ---------------------------------------------------------
 * Many independent 2D grids (jacobi-2d, poisson-2d Jacobi sweep with RHS,
 * gradient-2d) of uneven sizes and step counts, each with its own
 * (T, block_x in {16, 32, 64} x 256/block_x threads, E in {1, 2, 4}), run as
 * ONE persistent kernel launch captured in a CUDA graph.  No reference
 * counterpart: the reference runs one grid per process
 * (opencl/jacobi-2d/jacobi-2d.cpp:553-1048).  `grids` uses ots_params; the
 * fields read are stencil, problem_size, time_steps, time_tile, block_x,
 * elements_per_thread, coef and h2 (Poisson uses OTS_VARIANT_BASELINE). */
typedef struct ots_batch ots_batch;

ots_status ots_batch_create(const ots_params* grids, int32_t n, int32_t device, ots_batch** out);
void ots_batch_destroy(ots_batch* batch);
/* Total grid-point updates of one run, queue items, persistent CTAs. */
ots_status ots_batch_info(const ots_batch* batch, int64_t* updates, int32_t* items,
                          int32_t* ctas);
/* Dense n x n interior arrays (x fastest); aux is Poisson's f (else NULL). */
ots_status ots_batch_upload(ots_batch* batch, int32_t grid, const float* state, const float* aux);
ots_status ots_batch_download(ots_batch* batch, int32_t grid, float* state);
/* One graph launch running every grid to its step count. */
ots_status ots_batch_run(ots_batch* batch, ots_timing* timing);
ots_status ots_batch_run_async(ots_batch* batch);
ots_status ots_batch_stream(const ots_batch* batch, void** cuda_stream);
/* Limit of each item's bounded wait for its grid's previous chunk (2 s by
 * default); a wait that runs out makes ots_batch_run return
 * OTS_ERR_TIMEOUT.  Test hook: ots_batch_debug_hold(batch, g) makes every
 * later chunk of grid g wait for a completion count that is never reached
 * (-1 releases it).  No reference counterpart. */
ots_status ots_batch_set_wait_limit(ots_batch* batch, double seconds);
ots_status ots_batch_debug_hold(ots_batch* batch, int32_t grid);
/* Comparator on the same buffers: the grids one after another with one
 * launch per step (OTS_KERNEL_PLAIN) or per T steps (OTS_KERNEL_TILE). */
ots_status ots_batch_run_sequential(ots_batch* batch, int32_t kernel, ots_timing* timing);

/* ---- learned cost model --------------------------------------------------
 * A multi-layer perceptron (n_in -> hidden x (layers-1), SiLU -> 1) trained
 * and evaluated on the GPU by the library's own kernels.  It replaces the
 * reference's Weka k-NN cost model (scripts/run-weka.py:49-150, features from
 * scripts/extract-features.py:40-127): trained on measured sweeps, it ranks a
 * configuration space so that only the top k need measuring. */
typedef struct ots_mlp ots_mlp;

ots_status ots_mlp_create(int32_t n_in, int32_t hidden, int32_t layers, uint64_t seed,
                          int32_t device, ots_mlp** out);
void ots_mlp_destroy(ots_mlp* model);
ots_status ots_mlp_num_params(const ots_mlp* model, int64_t* n);
/* Parameters, layer by layer: W (out x in, row-major) then b (out). */
ots_status ots_mlp_get_params(const ots_mlp* model, float* params);
ots_status ots_mlp_set_params(ots_mlp* model, const float* params);
/* Inputs are standardised as (x - mean) * inv_std; targets as (y - y_mean) / y_std. */
ots_status ots_mlp_set_normalization(ots_mlp* model, const float* mean, const float* inv_std,
                                     float y_mean, float y_std);
/* Mean squared error on the standardised targets of n rows (n <= 4096) and
 * its gradient with respect to every parameter (grad may be NULL). */
ots_status ots_mlp_loss_grad(ots_mlp* model, const float* X, const float* y, int32_t n,
                             float* loss, float* grad);
/* AdamW minibatch training; each epoch is one replay of a captured CUDA
 * graph.  final_loss = mean minibatch loss of the last epoch. */
ots_status ots_mlp_train(ots_mlp* model, const float* X, const float* y, int32_t n,
                         int32_t epochs, int32_t batch, float lr, float weight_decay,
                         uint64_t seed, float* final_loss);
ots_status ots_mlp_predict(ots_mlp* model, const float* X, int32_t n, float* y_out);
/* Indices of the k largest predictions, best first. */
ots_status ots_mlp_topk(ots_mlp* model, const float* X, int32_t n, int32_t k, int32_t* idx_out);

/* Cost-model inference that allocates nothing -- no counterpart in the
 * reference.  For callers that must not call cudaMalloc while they pick
 * configurations: an application that hands out all device memory from its
 * own pool and does not let libraries allocate behind its back, or code that
 * runs where an allocation could block or fail at the wrong moment.  X
 * (n x n_in, row-major) and y (n) are DEVICE pointers the caller
 * owns; the work is enqueued on `cuda_stream` (a cudaStream_t, NULL for the
 * default stream) and this call does not wait for it.
 *   - The activations live in one fixed 2 MiB array compiled into libots
 *     (every GPU that loads the library holds it until the process exits):
 *     at most 4096 rows per call, and every layer at most 64 wide; larger
 *     requests are rejected with OTS_ERR_INVALID_ARGUMENT / UNSUPPORTED.
 *   - The first call on each device looks up that array's device address
 *     (cudaGetSymbolAddress) with the model's device current, and later calls
 *     reuse it.
 *   - All calls share the array: calls whose work overlaps on the GPU race
 *     (serialise them on one stream).  Each call overwrites what it reads,
 *     so nothing carries over from the previous call.
 *   - The model's device must be the current device. */
ots_status ots_mlp_predict_noalloc(const ots_mlp* model, const float* X, int32_t n, float* y,
                                   void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* OTS_H */
