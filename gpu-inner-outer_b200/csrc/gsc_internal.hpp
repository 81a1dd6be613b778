// gsc_internal.hpp -- host-side objects behind the C ABI handles, shared by
// the plain API (gsc_api.cu), the batched instances (gsc_batch.cu) and the
// serving loop (gsc_server.cu).
#pragma once

#include <array>
#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gsc_b200.h"
#include "gsc_kernels.cuh"
#include "gsc_pool.hpp"

// Device memory regions carved up by a RangePool.  `slab_bytes` > 0 lets the
// pool add regions of at least that size on demand; `cap` bounds the total
// (0 = no bound besides the context's budget).
struct DevicePool {
    struct Slab {
        char* base = nullptr;
        uint64_t bytes = 0;
        gsc_b200::RangePool ranges;
    };
    gsc_context* ctx = nullptr;
    std::vector<Slab> slabs;
    uint64_t slab_bytes = 0;
    uint64_t cap = 0;
    uint64_t total = 0;
    std::mutex mu;

    DevicePool(gsc_context* c, uint64_t slab, uint64_t capacity) : ctx(c), slab_bytes(slab), cap(capacity) {}
    ~DevicePool();
    // One region of exactly `bytes` now (a fixed pool); false when the device
    // or the context budget refuses it.
    bool reserve(uint64_t bytes);
    void* alloc(uint64_t bytes);   // nullptr when no region fits and none may be added
    void release(void* p, uint64_t bytes);
    uint64_t used();
    void trim();   // frees the regions nothing is allocated from
};

struct gsc_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    uint64_t budget = 0;
    std::atomic<uint64_t> in_use{0};
    std::mutex mem_mu;   // budget check + in_use update
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // Events of profiled solves and set-up uploads (created at first use).
    cudaEvent_t pev[gsc_b200::kProfileEvents] = {};
    int sm_count = 0;
    std::unique_ptr<DevicePool> pool;   // caching pool of the context's problems and abstractions
    // Streams for the set-up of batch instances (created at the first batch,
    // highest stream priority) and events to join them into `stream`.
    static constexpr int kSetupStreams = 8;
    cudaStream_t setup[kSetupStreams] = {};
    cudaEvent_t setup_ev[kSetupStreams + 1] = {};
    // Pinned host blocks of finished batches, kept for the next ones
    // (size -> block): freeing pinned memory costs far more host time than
    // taking a cached block.  Freed by gsc_context_trim and at destruction.
    std::mutex pin_mu;
    std::multimap<size_t, void*> pin_free;
    // Host-loop solves: a page-locked word, mapped for the device, into which
    // each iteration's last kernel writes iter | stop << 32, so that the host
    // follows the solve without copies in the stream (created at first use).
    unsigned long long* loop_word = nullptr;
    unsigned long long* loop_word_dev = nullptr;
};

struct gsc_abstraction {
    gsc_context* ctx = nullptr;
    gsc_b200::GridInfo g{};
    gsc_model_desc model{};
    double* xn = nullptr;
    double* yn = nullptr;
    double* thf = nullptr;
    double* vf = nullptr;
    DevicePool* pool = nullptr;                        // nullptr: cudaMalloc'd
    std::vector<std::pair<void*, uint64_t>> allocs;
    uint64_t bytes = 0;
    double build_ms = 0.0;
    double h2d_ms = 0.0;         // uploads of the trajectory tables
    bool sync_release = false;   // wait for the context stream before the memory is reused
    ~gsc_abstraction();
};

struct gsc_problem {
    gsc_context* ctx = nullptr;
    const gsc_abstraction* abs = nullptr;
    gsc_b200::GridInfo g{};
    gsc_b200::QueryInfo q{};
    uint32_t method = 0;          // requested, then the one chosen
    DevicePool* pool = nullptr;   // nullptr: every buffer cudaMalloc'd
    cudaStream_t stream = nullptr;
    bool sync_release = false;    // wait for `stream` before the memory is reused
    std::vector<std::pair<void*, uint64_t>> allocs;
    uint64_t bytes = 0;
    // masks and tables
    uint8_t* valid = nullptr;
    uint8_t* cand = nullptr;
    uint8_t* safe = nullptr;
    int safe_rank = 0;
    double* obstacles = nullptr;
    unsigned long long* counts = nullptr;   // [0] valid [1] cand [2] cand-not-valid [3] valid pairs [4] valid!=safe
    unsigned int* flags = nullptr;
    uint32_t *xt = nullptr, *yt = nullptr, *zt = nullptr, *wt = nullptr;
    int32_t* unsafe2 = nullptr;
    int32_t* unsafe4 = nullptr;
    int32_t* pvalid = nullptr;
    // the set-up plan (counts, flags, dilation widths), written by the device
    gsc_b200::PlanRecord* dplan = nullptr;
    gsc_b200::PlanRecord* hplan = nullptr;   // host copy (caller-provided pinned memory, or hplan_own)
    gsc_b200::PlanRecord hplan_own{};
    // Device address of *hplan when it is pinned host memory: the plan is then
    // stored there by a kernel, not copied by a copy engine (whose queue may
    // hold large result copies).
    gsc_b200::PlanRecord* hplan_dev = nullptr;
    bool fused_candidate = false;
    // stored
    uint2* boxes = nullptr;
    uint64_t S_pad = 0;
    uint4* boxes16 = nullptr;     // wide grids (a dimension of more than 255 cells)
    bool wide = false;
    int32_t* pd = nullptr;
    uint8_t* reach8 = nullptr;
    // fused
    gsc_b200::bword *validb = nullptr, *unsafeb = nullptr, *srcb = nullptr, *candb = nullptr, *dp = nullptr;
    gsc_b200::bword *reach0 = nullptr, *reach1 = nullptr, *active = nullptr, *hit = nullptr;
    uint32_t* best = nullptr;
    gsc_b200::bword* xcls = nullptr;
    uint8_t* xrep = nullptr;
    uint32_t max_reps = 0;
    gsc_b200::bword *dzw = nullptr, *vzw = nullptr;
    uint32_t* rowlost = nullptr;
    // sharded solve (gsc_problem_shard_*): this rank's slices and iterations done
    uint32_t shard_begin = 0, shard_slices = 0, shard_iter = 0;
    bool shard_stopped = false;
    uint32_t rl_words = 0;
    uint32_t* offz = nullptr;   // per omega column and theta cell: part of a dilated row's offset
    uint32_t* offv = nullptr;   // per acceleration and v cell: the other part
    uint8_t *kidx = nullptr, *lidx = nullptr;
    gsc_b200::DilateArgs dil{};
    int need_valid = 0;
    // common fixpoint state
    // The context's mirror word while a host-loop solve runs, else nullptr.
    unsigned long long* mirror = nullptr;
    uint32_t* controller = nullptr;
    uint32_t* reach_step = nullptr;
    gsc_b200::FixControl* fc = nullptr;
    unsigned long long* stats = nullptr;
    uint32_t stats_cap = 0;
    uint64_t valid_count = 0, candidate_count = 0, valid_pairs = 0;
    // graph
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    gsc_timings timings{};
    // Per-phase device times (gsc_problem_phase_timings).  h2d_ms: uploads of
    // the query's host arrays at creation; the rest from the last
    // GSC_SOLVE_PROFILE solve: prefix passes, satisfaction, reduction
    // (control or finalize kernel) and stop-record reads, summed, and per
    // iteration {iteration, prefix build, satisfaction, reduction incl. the
    // stop-record read}.
    bool time_h2d = false;
    double h2d_ms = 0.0;
    double pass_ms[4] = {0, 0, 0, 0};
    double prof_sat_ms = 0.0, prof_reduce_ms = 0.0, prof_memcpy_ms = 0.0;
    std::vector<std::array<float, 4>> iter_prof;
    uint64_t peak_used = 0;      // device memory in use on the GPU when last sampled
    ~gsc_problem();
};

namespace gsc_api {

inline int fail(gsc_context* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

#define GSC_CU(ctx, expr)                                                                              \
    do {                                                                                               \
        cudaError_t e__ = (expr);                                                                      \
        if (e__ != cudaSuccess) {                                                                      \
            return ::gsc_api::fail((ctx),                                                              \
                                   e__ == cudaErrorMemoryAllocation ? GSC_ERR_OUT_OF_MEMORY : GSC_ERR_CUDA, \
                                   std::string(#expr) + ": " + cudaGetErrorString(e__));               \
        }                                                                                              \
    } while (0)

#define GSC_TRY(expr)                  \
    do {                               \
        int s__ = (expr);              \
        if (s__ != GSC_OK) return s__; \
    } while (0)

int grid_from_model(const gsc_model_desc* m, gsc_b200::GridInfo* g, std::string* err);

// Device memory for a handle: from `pool` when set, else cudaMalloc under
// the context's budget.  Recorded in `allocs` and released by the owner.
int device_alloc(gsc_context* ctx, DevicePool* pool, std::vector<std::pair<void*, uint64_t>>& allocs,
                 uint64_t& bytes, void** p, uint64_t nbytes);
void device_release_all(gsc_context* ctx, DevicePool* pool, std::vector<std::pair<void*, uint64_t>>& allocs,
                        uint64_t& bytes);

// Pinned (page-locked, mapped) host memory through the context's cache: a
// cached block of at least `bytes` and at most twice that (plus 64 KB) is
// taken before a new one is allocated.  A block goes back with pinned_put
// once no device work uses it any more; the cache keeps at most
// kPinnedCacheMax bytes.
constexpr size_t kPinnedCacheMax = size_t(256) << 20;
cudaError_t pinned_get(gsc_context* ctx, size_t bytes, void** p, size_t* got);
void pinned_put(gsc_context* ctx, void* p, size_t bytes);
void pinned_trim(gsc_context* ctx);

template <typename T>
int palloc(gsc_problem* p, T** out, uint64_t count) {
    void* q = nullptr;
    const int s = device_alloc(p->ctx, p->pool, p->allocs, p->bytes, &q, count * sizeof(T));
    *out = static_cast<T*>(q);
    return s;
}

// Abstraction set-up without a host wait: tabulates the theta / v
// trajectories, uploads them and launches the nominal-successor kernel on
// `st`.  The three temporary tables are returned in `tmp` (owned by the
// caller until the stream has passed the kernel).
// h2d_ev (optional, 2 events) is recorded around the uploads.
int abstraction_enqueue(gsc_abstraction* a, cudaStream_t st, std::vector<std::pair<void*, uint64_t>>& tmp,
                        cudaEvent_t* h2d_ev = nullptr);

// Problem set-up in three steps:
//   stage1  masks, per-axis boxes and (for the fused method) the x classes,
//           plane representatives and the set-up plan, ending with the copy
//           of the plan record to p->hplan -- no host wait;
//   plan    (after the stream has passed stage1) chooses the method from the
//           plan record and checks the candidate set;
//   stage2  fixpoint buffers and the method's tables -- no host wait.
int problem_stage1(gsc_problem* p, const gsc_query_desc* qd);
int problem_plan(gsc_problem* p);
int problem_stage2(gsc_problem* p);

gsc_b200::FusedFixArgs fused_args(const gsc_problem* p, cudaGraphConditionalHandle cond, int use_cond);
int sm_count(gsc_context* ctx);
bool stored_fits(const gsc_b200::GridInfo& g);

// Batched execution of fused problems (gsc_batch.cu).
gsc_b200::InstanceDesc make_instance(const gsc_problem* p);
size_t instance_smem(const gsc_problem* p);
// Host work list [slot | sat_off | dil_off | fin_off | ini_off] of probs[k]
// placed at slots[k].
void build_work_list(const std::vector<const gsc_problem*>& probs, const std::vector<uint32_t>& slots,
                     uint32_t chunk, std::vector<uint32_t>& buf, gsc_b200::WorkTotals& tot);
gsc_b200::WorkList device_work_list(const uint32_t* dbuf, uint32_t n, uint32_t chunk, gsc_b200::FixControl* status,
                                    uint32_t* running);
// Register words of the batched satisfaction kernel for rows of w words.
uint32_t wmax_of(uint32_t w);

}  // namespace gsc_api
