/*
 * gsc_b200.h -- C ABI of the B200 (sm_100a) grid symbolic-control library.
 *
 * The reference (zzx-ur/gpu-inner-outer, namespace gsc) exposes its CUDA
 * backend as two C++ functions, include/gsc/cuda_api.hpp:87-88:
 *
 *     bool gsc::cuda_backend_compiled();
 *     gsc::GpuRunReport gsc::run_case_cuda_u32(const gsc::CaseConfig&);
 *
 * run_case_cuda_u32 (cuda/kernels.cu:492-875) builds the masks on the host,
 * launches abstraction_kernel (:164-217), then loops over fixpoint iterations
 * (:654-767) of build_prefix_on_device (:403-484), pair_satisfaction_kernel
 * (:310-336) and reduce_inputs_kernel (:338-393), and copies everything back.
 *
 * This header splits that call into device-resident stages behind plain C
 * types (no C++ or torch types cross the boundary):
 *
 *   gsc_abstraction_*  the dynamics part of abstraction_kernel: nominal Euler
 *                      successors of every (cell, input), kept on the device;
 *   gsc_problem_*      one K-invariance query against a resident abstraction:
 *                      masks, quantised successor boxes, and the fixpoint;
 *   gsc_run_case       the whole reference call in one step;
 *   gsc_batch_*        many independent instances solved together (no
 *                      counterpart in the reference);
 *   gsc_server_*       a request loop of K-invariance queries against
 *                      resident abstractions (no counterpart in the reference).
 *
 * Every entry point returns a gsc_status.  Results go to caller-provided host
 * buffers.  Device memory is owned by the handles.  There is no CPU fallback:
 * without a usable CUDA device the calls fail with GSC_ERR_NO_DEVICE.
 */
#ifndef GSC_B200_H
#define GSC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSC_B200_ABI_VERSION 1

typedef enum {
    GSC_OK = 0,
    GSC_ERR_INVALID_ARGUMENT = 1,   /* bad grid, bad pointer, bad option          */
    GSC_ERR_CUDA = 2,               /* a CUDA runtime call failed                 */
    GSC_ERR_OUT_OF_MEMORY = 3,      /* device allocation failed or over budget    */
    GSC_ERR_UNSUPPORTED = 4,        /* valid input outside what a method handles  */
    GSC_ERR_NO_DEVICE = 5,          /* no CUDA device (kernels.cu:497-502)        */
    GSC_ERR_CANDIDATE_INVALID = 6,  /* candidate set contains invalid states
                                       (abstraction.hpp:268-272)                  */
    GSC_ERR_TIMEOUT = 7             /* a bounded device-side wait ran out         */
} gsc_status;

/* Fixpoint outcome, reachability.hpp:133-152 (messages kept verbatim by
 * gsc_message_string). */
enum {
    GSC_MSG_NONE = 0,
    GSC_MSG_CONVERGED = 1,          /* "all candidate states obtained a controller"  */
    GSC_MSG_STALLED = 2,            /* "iteration stalled before candidate closure"  */
    GSC_MSG_MAX_ITERATIONS = 3      /* "maximum iterations reached"                  */
};

/* State constraint kinds: ConstraintType (config.hpp:19-24) plus the quadric
 * safe set (x*x)*qa - (y*y)*qb <= c && fabs(y) <= ymax, which the reference can
 * only state as kCustom. */
enum {
    GSC_CONSTRAINT_NONE = 0,        /* params unused                              */
    GSC_CONSTRAINT_HYPERBOLIC = 1,  /* a, b, c: x^2 - y^2 <= a && b*y^2 - x^2 <= c */
    GSC_CONSTRAINT_ELLIPTIC = 2,    /* a, b: (x/a)^2 + (y/b)^2 <= 1                */
    GSC_CONSTRAINT_QUADRIC = 3      /* qa, qb, c, ymax                             */
};

enum {
    GSC_CANDIDATE_RECT = 0,         /* candidate[0..3] lb, [4..7] ub, inclusive     */
    GSC_CANDIDATE_ELLIPSE = 1       /* cx, cy, wx, wy, r2; intersected with valid  */
};

/* Solve methods.  Both give bit-identical results. */
enum {
    GSC_METHOD_AUTO = 0,            /* FUSED when it applies, else STORED          */
    GSC_METHOD_STORED = 1,          /* per-pair int32 index boxes in HBM, int32 4-D
                                       prefix scan, 16-corner box count            */
    GSC_METHOD_FUSED = 2            /* boxes recomputed from per-axis tables inside
                                       the satisfaction kernel, bit-sliced sets    */
};

/* Solve flags. */
enum {
    GSC_SOLVE_GRAPH = 1u << 0,      /* run the fixpoint as one CUDA graph with a
                                       device-side while condition (instantiated
                                       at a problem's first such solve, about
                                       0.3 ms on a B200)                          */
    GSC_SOLVE_PROFILE = 1u << 1     /* host loop, one iteration at a time, CUDA
                                       events around the scan and satisfaction
                                       kernels (gsc_timings.*_kernel_ms)           */
};

/* The grid and dynamics (CaseConfig fields that the successor boxes' nominal
 * part depends on, config.hpp:41-66; grids grid.hpp:103-168; model
 * model.hpp:8-112). */
typedef struct {
    double state_lb[4];
    double state_ub[4];
    double state_eta[4];
    int32_t wrap_dim;               /* must be 2 (theta), as in all reference cases */
    double input_lb[2];
    double input_ub[2];
    double input_eta[2];
    double sample_time;
    uint32_t integration_substeps;
} gsc_model_desc;

/* One K-invariance query (the rest of CaseConfig). */
typedef struct {
    double disturbance_half_width[4];
    int32_t constraint_kind;
    double constraint_params[4];
    double map_lb[4];
    double map_ub[4];
    uint32_t obstacle_count;
    const double* obstacles;        /* obstacle_count x {lb[4], ub[4]}            */
    int32_t candidate_kind;
    double candidate[8];
    uint32_t max_iterations;
    /* Optional host masks replacing the ones built from the description above
     * (NULL = build on the device).  safe_mask is the state constraint
     * evaluated at cell centres: rank 2 = [ny][nx] over (x, y), rank 4 = one
     * byte per state.  When given it replaces constraint_kind everywhere: in the
     * valid mask, at the source state and over every successor box.  A custom
     * constraint (ConstraintType::kCustom) is passed this way. */
    const uint8_t* safe_mask;
    int32_t safe_mask_rank;
    const uint8_t* valid_mask;      /* one byte per state                         */
    const uint8_t* candidate_mask;  /* one byte per state                         */
} gsc_query_desc;

/* Outputs.  Buffers are caller-owned host memory; any may be NULL. */
typedef struct {
    uint8_t* valid_mask;            /* [states]                                   */
    uint8_t* candidate_mask;        /* [states]                                   */
    uint8_t* reachable_mask;        /* [states]                                   */
    uint32_t* controller;           /* [states], 0xFFFFFFFF = none (types.hpp:22)  */
    uint32_t* reach_step;           /* [states], 0xFFFFFFFF = unreachable         */
    uint64_t* iter_new_reachable;   /* [iter_capacity]                            */
    uint64_t* iter_new_certified;   /* [iter_capacity]                            */
    uint32_t iter_capacity;
    /* Filled by the library. */
    uint32_t shape[4];
    uint32_t input_shape[2];
    uint64_t states;
    uint64_t inputs;
    uint64_t pairs;
    uint32_t iterations;
    int32_t converged;
    int32_t message;                /* GSC_MSG_*                                  */
    uint64_t reachable_states;
    uint64_t certified_candidates;
    uint64_t candidate_count;
    uint64_t valid_count;
} gsc_result;

/* Device timings of the last solve, CUDA events on the library's stream. */
typedef struct {
    double abstraction_ms;          /* gsc_abstraction_create kernels             */
    double prepare_ms;              /* masks + boxes (gsc_problem_create)         */
    double solve_ms;                /* the fixpoint                               */
    double readback_ms;             /* gsc_problem_read copies                    */
    uint64_t device_bytes;          /* device memory held by the problem          */
    uint32_t method;                /* method actually used                       */
    uint32_t kernel_launches;       /* kernels launched by the last solve         */
    uint32_t iterations;            /* fixpoint iterations of the last solve      */
    uint32_t sat_launches;          /* satisfaction-kernel launches timed         */
    double sat_kernel_ms;           /* GSC_SOLVE_PROFILE: satisfaction kernels    */
    double scan_kernel_ms;          /* GSC_SOLVE_PROFILE: set / prefix rebuilds
                                       (fused: the (theta, v) dilation)           */
    uint64_t pair_tests;            /* stored: boxes streamed; fused: (state,
                                       input) tests, summed over iterations       */
    uint64_t aux_count;             /* stored: box counts evaluated; fused:
                                       (slice, representative input) planes
                                       staged, summed over iterations             */
    uint32_t sat_threads;           /* fused: threads per satisfaction block      */
    uint32_t max_reps;              /* fused: most representative accelerations
                                       of one omega column                        */
} gsc_timings;

typedef struct gsc_context gsc_context;
typedef struct gsc_abstraction gsc_abstraction;
typedef struct gsc_problem gsc_problem;

/* Replaces gsc::cuda_backend_compiled() (cuda_api.hpp:87). */
int gsc_cuda_backend_compiled(void);

int gsc_abi_version(void);
const char* gsc_status_string(int status);
/* reachability.hpp:135,140,151 */
const char* gsc_message_string(int message);

/* Grid shapes exactly as build_state_grid / build_input_grid
 * (grid.hpp:103-168): shape = (uint32_t)ceil(width / eta). */
int gsc_grid_shape(const gsc_model_desc* model, uint32_t shape[4], uint32_t input_shape[2]);

/* A context binds a device and a stream (NULL stream = a private stream).
 * A context and the handles made from it are used from one host thread at
 * a time (its timing events and its host-loop stop word are its own);
 * threads that solve at the same time use a context each.  gsc_run_case
 * keeps one context per device and serialises its calls; the gsc_server_*
 * calls are thread-safe.
 * Mirrors the device checks of kernels.cu:496-502.  Problems and
 * abstractions of a context take their device memory from the context's
 * caching pool (regions of 64 MB or more, sub-allocated first-fit), so a
 * create / destroy cycle costs no cudaMalloc / cudaFree once warm; memory
 * returns to the driver at gsc_context_trim or gsc_context_destroy. */
int gsc_context_create(int device, void* cuda_stream, gsc_context** out);
/* Destroy every problem, abstraction, batch and server of a context before
 * the context. */
void gsc_context_destroy(gsc_context* ctx);
const char* gsc_last_error(const gsc_context* ctx);
/* Device memory the context may hold: its pool regions plus batches and
 * servers (0 = no limit).  Creation fails with GSC_ERR_OUT_OF_MEMORY beyond it. */
int gsc_context_set_memory_budget(gsc_context* ctx, uint64_t bytes);
/* Device memory the context holds now (pool regions, in use or cached). */
uint64_t gsc_context_memory_in_use(const gsc_context* ctx);
/* Returns the pool regions no handle uses to the driver, and the pinned host
 * blocks that destroyed batches left in the context's cache for reuse. */
int gsc_context_trim(gsc_context* ctx);

/* The nominal successor tables of abstraction_kernel (kernels.cu:164-217,
 * model.hpp:26-46) for every (cell, input), built once and kept resident. */
int gsc_abstraction_create(gsc_context* ctx, const gsc_model_desc* model, gsc_abstraction** out);
void gsc_abstraction_destroy(gsc_abstraction* abs);

/* Prepare a query: masks (abstraction.hpp:65-106), quantised successor boxes
 * with constraint and bounds validity (abstraction.hpp:161-209,
 * grid.hpp:181-251), and the fixpoint state (reachability.hpp:36-51).
 * method = GSC_METHOD_*. */
int gsc_problem_create(gsc_context* ctx, const gsc_abstraction* abs, const gsc_query_desc* query,
                       uint32_t method, gsc_problem** out);
void gsc_problem_destroy(gsc_problem* p);

/* Run the fixpoint (kernels.cu:650-767 / reachability.hpp:53-153) on the
 * device.  Resets the fixpoint state first, so a problem can be solved again.
 * Returns when the solve has finished (its device time in
 * gsc_timings.solve_ms).  Without GSC_SOLVE_GRAPH the host queues the
 * iterations, two ahead of the last one finished, which it learns from a
 * word of mapped host memory that each iteration's last kernel writes. */
int gsc_problem_solve(gsc_problem* p, uint32_t flags);

/* Copy the results into caller buffers (kernels.cu:776-832).  Synchronises. */
int gsc_problem_read(gsc_problem* p, gsc_result* out);

/* The reference's abstraction arrays (cuda_api.hpp:82-84: min_flat, max_flat,
 * valid; pair = state * inputs + input), produced on demand.  Synchronises. */
int gsc_problem_export_abstraction(gsc_problem* p, uint32_t* min_flat, uint32_t* max_flat, uint8_t* valid);

int gsc_problem_timings(const gsc_problem* p, gsc_timings* out);

/* Per-phase device times and memory of a problem in the terms of the
 * reference's report: the fields of KernelTimings and GpuMemoryStats
 * (include/gsc/cuda_api.hpp:24-58), which cuda/kernels.cu fills with CUDA
 * events around each launch (kernels.cu:403-484, :605-640, :654-767,
 * :785-851).  Set-up and readback times come from gsc_abstraction_create,
 * gsc_problem_create and the last gsc_problem_read; the kernel breakdown
 * from the last solve run with GSC_SOLVE_PROFILE (zero after any other
 * solve).  The prefix build has no separate scatter: the set is read inside
 * its first pass. */
typedef struct {
    double abstraction_kernel_ms;     /* abstraction tables + the problem's mask and box kernels      */
    double abstraction_memcpy_h2d_ms; /* set-up uploads: trajectory tables, host masks, obstacles      */
    double scatter_mask_ms;           /* 0: folded into the first prefix pass                          */
    double scan_axis_ms[4];           /* stored: prefix passes in launch order (a two-pass build:
                                         [0] x and y, [1] theta and v); fused: [0] = the (theta, v)
                                         dilation of D'                                                */
    double prefix_build_total_ms;     /* sum of scan_axis_ms                                           */
    double pair_satisfaction_ms;      /* satisfaction kernels (exists-input reduction fused in)        */
    double reduce_inputs_ms;          /* stored: control kernel; fused: finalize kernel                */
    double iteration_memcpy_ms;       /* the host loop's reads of the stop record                      */
    double result_memcpy_d2h_ms;      /* last gsc_problem_read                                         */
    double total_kernel_ms;           /* abstraction + prefix + satisfaction + reduction (kernels.cu:841-845) */
    double total_memcpy_ms;           /* h2d + iteration + result copies (kernels.cu:846-849)          */
    double total_compute_ms;          /* kernel + memcpy (kernels.cu:850-851)                          */
    uint64_t total_allocated_bytes;   /* device memory of the abstraction and the problem              */
    uint64_t peak_usage_bytes;        /* device memory in use on the GPU (cudaMemGetInfo), highest
                                         sample taken by this call on the problem                      */
    uint64_t abstraction_bytes;       /* abstraction tables + the problem's boxes, classes, safe tables */
    uint64_t prefix_bytes;            /* stored: prefix tables; fused: D' and its dilated copies       */
    uint64_t iteration_bytes;         /* masks, sets, controller, reach_step, counters, control        */
    uint64_t result_bytes;            /* bytes a full gsc_problem_read copies to the host              */
    uint32_t profiled_iterations;     /* iterations with per-iteration times                           */
} gsc_phase_timings;

int gsc_problem_phase_timings(const gsc_problem* p, gsc_phase_timings* out);

/* Per-iteration device times of the last GSC_SOLVE_PROFILE solve, the time
 * fields of IterationStats (cuda_api.hpp:11-21): entry i is iteration i + 1
 * (capacity entries at most; gsc_phase_timings.profiled_iterations exist).
 * iteration = prefix build + satisfaction + reduction; reduction includes the
 * host loop's read of the stop record, as the reference's reduction_ms
 * includes its counter copies (kernels.cu:687-721).  Any pointer may be NULL. */
int gsc_problem_iteration_timings(const gsc_problem* p, uint32_t capacity, double* iteration_ms,
                                  double* prefix_build_ms, double* satisfaction_ms, double* reduction_ms);

/* Replaces gsc::run_case_cuda_u32 (cuda_api.hpp:88, kernels.cu:492-875):
 * abstraction, query, fixpoint and readback in one call on `device`.  For a
 * one-shot call, flags without GSC_SOLVE_GRAPH are the faster choice: the
 * graph's instantiation (about 0.3 ms on a B200) is paid by one solve only. */
int gsc_run_case(int device, const gsc_model_desc* model, const gsc_query_desc* query, uint32_t method,
                 uint32_t flags, gsc_result* out, gsc_timings* timings);

/* No counterpart in the reference.
 *
 * The backward-reachability fixpoint over an abstraction the caller already
 * holds in device memory, in the reference's layout (min_flat, max_flat and
 * valid per pair, pair = state * inputs + input), without allocating any
 * memory.  It is meant for callers that may not call cudaMalloc when they
 * need a solve: a process whose device memory is already carved into its own
 * pools, a plugin whose host owns every allocation, or a latency-critical path
 * that must not enter the driver's allocator (which can synchronise the device
 * and can fail).
 *
 * Every pointer except `summary` is device memory owned by the caller:
 * inputs min_flat, max_flat, pair_valid ([states * inputs]), valid_mask and
 * candidate_mask ([states]); outputs reachable_mask, controller, reach_step
 * ([states]).  `summary` (host, optional) receives the iteration count, stop
 * message and set sizes.  The working tables live in one fixed device array
 * inside the library (about 40 MiB, held by every GPU that loads the library
 * until the process exits).  Grids whose padded table
 * (nx+1)(ny+1)(ntheta+1)(nv+1) has more than 4,718,592 entries are refused
 * with GSC_ERR_OUT_OF_MEMORY before any device work, and so is a
 * `max_iterations` argument that, capped at states + 1, exceeds 4,094 (the
 * limit applies to the argument, not to the iterations a solve ends up
 * running).  A candidate set holding invalid states is refused with
 * GSC_ERR_CANDIDATE_INVALID, as the reference refuses it
 * (abstraction.hpp:268-272).  All calls share the array, so calls that
 * overlap on the GPU race: serialise them.  The first call on a device looks
 * the array's address up (cudaGetSymbolAddress) and keeps it for the life of
 * the process; make that first call before any stream capture, and do not call
 * this entry point on a device again after cudaDeviceReset of that device.
 * When a launch or copy fails part-way the call first waits for the work it
 * had queued on `cuda_stream`, then returns GSC_ERR_CUDA.  Returns after
 * synchronising `cuda_stream`. */
int gsc_fixpoint_noalloc(const uint32_t shape[4], uint32_t inputs, int32_t wrap_dim, const uint32_t* min_flat,
                         const uint32_t* max_flat, const uint8_t* pair_valid, const uint8_t* valid_mask,
                         const uint8_t* candidate_mask, uint32_t max_iterations, uint8_t* reachable_mask,
                         uint32_t* controller, uint32_t* reach_step, gsc_result* summary, void* cuda_stream);

/* ---- Sharded fixpoint: one problem over several GPUs ----------------------
 * No counterpart in the reference (which runs on one GPU).  G ranks, one
 * process per GPU, each hold the whole problem (its own context, abstraction
 * and problem, created alike) and iterate only their own contiguous range of
 * (theta, v) slices [slice_begin, slice_end).  States are x-fastest, so a
 * slice range is one contiguous slab of every state array, and of the
 * bit-sliced D' words (words_per_slice words per slice).  Per iteration each
 * rank calls gsc_problem_shard_step (the dilation of D' over the whole grid,
 * then the satisfaction test, the exists-input reduction and the finalize of
 * its own slices; counts[] = its newly reachable and newly certified
 * states), the ranks all-gather their slabs of D' in place
 * (gsc_problem_shard_words: device memory, slab k at word
 * slice_begin_k * words_per_slice) and sum their counts, and every rank
 * applies the stop rules with the sums (gsc_problem_shard_control, the
 * reference's rules of reachability.hpp:133-144).  Every iteration of a
 * sharded solve tests every pair (no row-lost skipping).  After the stop,
 * gsc_problem_read gives the global iteration count, stop message and set
 * sizes, and the rank's own slab of every state array; the caller gathers
 * the slabs.  Fused method only; gsc_problem_solve ends the sharding. */
int gsc_problem_shard_begin(gsc_problem* p, uint32_t slice_begin, uint32_t slice_end);
int gsc_problem_shard_step(gsc_problem* p, uint64_t counts[2]);
int gsc_problem_shard_words(const gsc_problem* p, void** dprime_words, uint64_t* words_per_slice);
/* *stop = 1 once a stop rule has fired (then further steps do nothing). */
int gsc_problem_shard_control(gsc_problem* p, uint64_t new_reachable, uint64_t new_certified, int* stop);

/* ---- Closed-loop simulation of the controller ----------------------------
 * The consumer of the controller table, plots/postprocess_controller.py:66-224:
 * trajectories of the continuous unicycle under the problem's controller
 * (after gsc_problem_solve), one device thread per trajectory reading the
 * device-resident table.  Each sample period maps the state to a cell as
 * the script does (theta wrapped with atan2(sin, cos), round((x - lb) / eta)
 * half to even, clamped; :66-101), stops at the invalid input (:103-130),
 * and takes integration_substeps Euler substeps x + dt * (f(x, u) + w) with
 * theta re-wrapped (:132-176).  w is uniform in [-dhw, dhw] per dimension
 * and substep, drawn from Philox4x32-10 keyed by `seed` (counter: substep
 * and trajectory), so a run is reproducible; the script draws from numpy's
 * global generator instead.  x0: [count][4]; trajectories (optional):
 * [count][steps + 1][4], rows after a stop left 0 as in the script;
 * final_states (optional): [count][4]; steps_done (optional): [count]. */
int gsc_problem_simulate(gsc_problem* problem, uint32_t count, const double* x0, uint32_t steps, uint64_t seed,
                         double* trajectories, double* final_states, uint32_t* steps_done);

/* ---- Batched instances --------------------------------------------------
 * No counterpart in the reference (which solves one case per call).  Many
 * independent instances -- each its own model and query, of any grid and
 * input size the fused method takes -- are set up together and solved
 * together: every fixpoint iteration of every instance is one pass of four
 * kernels over all instances (persistent blocks walking a task list), and
 * with GSC_SOLVE_GRAPH the whole loop is one CUDA graph whose while-node
 * reads a device flag cleared when no instance is left running.  Device
 * memory comes from the context's caching pool.  Each instance's result is
 * bit-identical to its own gsc_problem solve.  Fused
 * method only: an instance the fused method cannot take fails the create
 * with GSC_ERR_UNSUPPORTED and the instance index in gsc_last_error. */
typedef struct gsc_batch gsc_batch;

typedef struct {
    uint32_t autotune;            /* 1: time launch shapes on this batch, keep the fastest
                                     (cached per batch shape class in the process)        */
    uint32_t sat_threads;         /* threads per satisfaction block: 64, 128, 256 (0 = 128)  */
    uint32_t sat_blocks_per_sm;   /* persistent satisfaction blocks per SM (0 = one block
                                     per task)                                             */
    uint32_t chunk_words;         /* word positions per dilate / finalize task (0 = 2048)  */
    uint32_t sat_warp_tasks;      /* 1: each warp of a satisfaction block runs its own task
                                     (sat_threads / 32 tasks per block, no block barriers);
                                     0: the whole block runs one task                       */
} gsc_batch_options;

typedef struct {
    double create_ms;             /* host wall clock of gsc_batch_create (set-up of all)   */
    double tune_ms;               /* of which autotuning trials                            */
    double solve_ms;              /* last gsc_batch_solve, device events                   */
    uint64_t device_bytes;        /* device memory held by the batch                       */
    uint32_t instances;
    uint32_t max_iterations_run;  /* most fixpoint iterations of one instance, last solve  */
    uint32_t kernel_launches;     /* kernels launched by the last solve                    */
    uint32_t sat_threads;         /* launch shapes in use                                  */
    uint32_t sat_blocks_per_sm;
    uint32_t chunk_words;
    uint32_t tuned;               /* 1 = shapes from trials, 2 = from the process cache    */
    uint32_t sat_warp_tasks;      /* as gsc_batch_options                                  */
    uint64_t pair_tests;          /* (state, input) tests of the last solve, all instances */
} gsc_batch_report;

int gsc_batch_create(gsc_context* ctx, uint32_t count, const gsc_model_desc* models, const gsc_query_desc* queries,
                     const gsc_batch_options* options, gsc_batch** out);
/* flags: GSC_SOLVE_GRAPH (else a host loop that checks the device flag). */
int gsc_batch_solve(gsc_batch* batch, uint32_t flags);
/* Instance `index` of the last solve, as gsc_problem_read. */
int gsc_batch_read(gsc_batch* batch, uint32_t index, gsc_result* out);
/* Every instance at once (out: one gsc_result per instance, in creation
 * order): all copies are queued, then one wait. */
int gsc_batch_read_all(gsc_batch* batch, gsc_result* out);
int gsc_batch_timings(gsc_batch* batch, gsc_batch_report* out);
void gsc_batch_destroy(gsc_batch* batch);
/* Sets up, solves and reads `count` instances in one call (no reference
 * counterpart), in parts of `part_instances` instances (0 = an eighth of
 * them) that overlap: while part k solves (graph), part k+1 is set up and
 * part k-1's results are copied into `results` (one gsc_result per
 * instance, in order, buffers as for gsc_batch_read_all).  With autotune
 * the first part chooses the launch shapes and the later parts reuse them.
 * Returns when every result is in host memory; each result equals the
 * instance's own gsc_problem solve.  A failing part fails the call, with
 * the part's instance range in gsc_last_error. */
int gsc_batch_run(gsc_context* ctx, uint32_t count, const gsc_model_desc* models, const gsc_query_desc* queries,
                  const gsc_batch_options* options, uint32_t part_instances, gsc_result* results);

/* ---- Serving loop ---------------------------------------------------------
 * No counterpart in the reference.  A loop thread serves K-invariance
 * queries (safe set, candidate set, disturbance bound, iteration cap: a
 * gsc_query_desc) against abstractions kept resident on the device.  Queries
 * are admitted in arrival order while a slot is free and their device memory
 * fits the server's budget; admitted queries are set up on a second stream
 * while the running ones iterate, and join the running set at the next
 * iteration step (continuous batching: every step runs one batched fixpoint
 * iteration -- or iterations_per_step -- of every running query in four
 * launches).  A query that stops leaves the set, its results are copied to
 * the caller's buffers on a third stream, and its memory and slot go to the
 * next query.  Each query's result is bit-identical to its own gsc_problem
 * solve (fused method).  All gsc_server_* calls are thread-safe. */
typedef struct gsc_server gsc_server;

typedef struct {
    uint64_t memory_budget;         /* device bytes for queries in flight (0 = half the free memory) */
    uint32_t max_slots;             /* queries on the device at once (0 = 256)                        */
    uint32_t iterations_per_step;   /* fixpoint iterations between host checks (0 = 2)               */
    uint32_t sat_threads;           /* as gsc_batch_options (0 = 64)                                  */
    uint32_t sat_blocks_per_sm;     /* (0 = 16)                                                       */
    uint32_t chunk_words;           /* (0 = 1024)                                                     */
    uint32_t sat_warp_tasks;        /* as gsc_batch_options (a step whose staging would not fit runs
                                       one task per block)                                            */
} gsc_server_options;

typedef struct {
    uint64_t submitted;
    uint64_t completed;             /* finished, successfully or not                */
    uint64_t failed;
    uint64_t queued;                /* waiting for admission                        */
    uint64_t in_flight;             /* admitted, not yet completed                  */
    uint64_t steps;                 /* batched iteration steps launched             */
    uint64_t max_running;           /* most queries iterating in one step           */
    uint64_t device_bytes_budget;
    uint64_t device_bytes_in_use;
    uint64_t peak_device_bytes;
} gsc_server_report;

int gsc_server_create(gsc_context* ctx, const gsc_server_options* options, gsc_server** out);
/* Queues one query against `abs` (an abstraction of the server's context).
 * The query's host arrays (obstacles, masks) and every buffer of `out` must
 * stay valid until the query completes; `out` is then filled as by
 * gsc_problem_read (result buffers in pinned host memory let the copies
 * overlap the device work).  *ticket identifies the query. */
int gsc_server_submit(gsc_server* server, const gsc_abstraction* abs, const gsc_query_desc* query,
                      gsc_result* out, uint64_t* ticket);
/* Waits for a ticket (timeout_ms < 0: no limit).  Returns GSC_ERR_TIMEOUT if
 * it has not completed in time, else GSC_OK with *status = the query's own
 * gsc_status and *latency_ms = submit-to-completion time; a completed ticket
 * is then forgotten (wait once per ticket). */
int gsc_server_wait(gsc_server* server, uint64_t ticket, int32_t timeout_ms, int* status, double* latency_ms);
int gsc_server_stats(gsc_server* server, gsc_server_report* out);
/* Completes every submitted query, then stops the loop and frees the server. */
void gsc_server_destroy(gsc_server* server);

#ifdef __cplusplus
}
#endif

#endif /* GSC_B200_H */
