// gsc_batch.cu -- batched instances (gsc_batch_* of include/gsc_b200.h).
//
// No counterpart in the reference, which runs one case per call
// (cuda/kernels.cu:492-875).  Set-up of N instances is the one-problem
// set-up run N times on one stream with a single host wait (for the N plan
// records) in the middle; all device memory comes from one growable pool.
// The fixpoint is the batched kernels of gsc_batch_kernels.cu over every
// instance, optionally as one CUDA graph: [init] -> while (any running)
// { dilate, satisfaction, finalize, status }.  An instance that fills the
// GPU on its own (is_big_instance) iterates with the one-problem kernels
// inside the same step and shares only init and status.  Launch shapes come
// from the options, or from a small autotuner that times candidate shapes
// on the batch's small instances and caches the winner per shape class.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "gsc_internal.hpp"

using namespace gsc_b200;
using namespace gsc_api;

namespace gsc_api {

InstanceDesc make_instance(const gsc_problem* p) {
    InstanceDesc d;
    std::memset(&d, 0, sizeof(d));
    d.g = p->g;
    d.a = fused_args(p, 0, 0);
    d.cand = p->cand;
    d.counts = p->counts;
    d.max_iterations = p->q.max_iterations;
    d.stats_cap = p->stats_cap;
    d.sat_tasks = p->g.slices * p->g.mw;
    d.words = static_cast<uint32_t>(p->g.rows * p->g.W);
    return d;
}

size_t instance_smem(const gsc_problem* p) {
    return fused_smem_bytes(p->g, class_words(p->g), p->need_valid, p->max_reps, false);
}

void build_work_list(const std::vector<const gsc_problem*>& probs, const std::vector<uint32_t>& slots,
                     uint32_t chunk, std::vector<uint32_t>& buf, WorkTotals& tot) {
    const size_t n = slots.size();
    buf.assign(n + 4 * (n + 1), 0);
    uint32_t* slot = buf.data();
    uint32_t* sat = slot + n;
    uint32_t* dil = sat + n + 1;
    uint32_t* fin = dil + n + 1;
    uint32_t* ini = fin + n + 1;
    for (size_t k = 0; k < n; ++k) {
        const gsc_problem* p = probs[k];
        const uint64_t words = p->g.rows * p->g.W;
        const uint64_t span = std::max<uint64_t>({words, p->g.S, static_cast<uint64_t>(kStatsCols) * p->stats_cap});
        slot[k] = slots[k];
        sat[k + 1] = sat[k] + p->g.slices * p->g.mw;
        dil[k + 1] = dil[k] + static_cast<uint32_t>((words + chunk - 1) / chunk);
        fin[k + 1] = fin[k] + static_cast<uint32_t>((words + chunk - 1) / chunk);
        ini[k + 1] = ini[k] + static_cast<uint32_t>((span + chunk - 1) / chunk);
    }
    tot.sat = sat[n];
    tot.dil = dil[n];
    tot.fin = fin[n];
    tot.ini = ini[n];
}

WorkList device_work_list(const uint32_t* dbuf, uint32_t n, uint32_t chunk, FixControl* status, uint32_t* running) {
    WorkList wl{};
    wl.slot = dbuf;
    wl.sat_off = dbuf + n;
    wl.dil_off = wl.sat_off + n + 1;
    wl.fin_off = wl.dil_off + n + 1;
    wl.ini_off = wl.fin_off + n + 1;
    wl.n = n;
    wl.chunk = chunk;
    wl.status = status;
    wl.running = running;
    return wl;
}

uint32_t wmax_of(uint32_t w) { return w <= 1 ? 1 : w == 2 ? 2 : w <= 4 ? 4 : 8; }

}  // namespace gsc_api

struct gsc_batch;
namespace {
void release_batch_graph(gsc_batch* b);
}

struct gsc_batch {
    gsc_context* ctx = nullptr;
    DevicePool* pool = nullptr;   // the context's caching pool
    std::vector<std::pair<void*, uint64_t>> own;   // instance table and work list
    uint64_t own_bytes = 0;
    std::vector<std::unique_ptr<gsc_abstraction>> abs;
    std::vector<std::unique_ptr<gsc_problem>> probs;
    PlanRecord* hplans = nullptr;   // pinned
    uint32_t* hrunning = nullptr;   // pinned
    FixControl* hfc = nullptr;      // pinned: every instance's control record, for reads (written by
                                    // the status kernel after every iteration)
    FixControl* hfc_dev = nullptr;  // its device address
    PlanRecord* hplans_dev = nullptr;
    unsigned long long* hstats = nullptr;   // pinned: every instance's per-iteration counters
    std::vector<uint64_t> stats_off;        // instance -> its first entry in hstats
    InstanceDesc* ddesc = nullptr;
    uint32_t* dlist = nullptr;       // the small instances' work list
    uint32_t* dlist_all = nullptr;   // every instance: init and status
    uint32_t* drunning = nullptr;
    std::vector<uint32_t> hlist, hlist_all;
    // Pinned staging of the instance table and the two work lists, so their
    // uploads do not wait for the set-up queued before them.
    InstanceDesc* hdesc_pin = nullptr;
    uint32_t* hlist_pin = nullptr;   // [2][count + 4 * (count + 1)]
    bool lists_uploaded = false;
    void* pin_early = nullptr;   // hplans, hrunning, hfc (from the context's pinned cache)
    void* pin_late = nullptr;    // hstats, hdesc_pin, hlist_pin (from the context's pinned cache)
    size_t pin_early_bytes = 0, pin_late_bytes = 0;
    // Between the two set-up phases (batch_begin, batch_finish): the
    // abstractions' temporary tables, the set-up streams in use and an
    // event per stream after its stage-1 work.
    std::vector<std::vector<std::pair<void*, uint64_t>>> setup_tmp;
    uint32_t setup_base = 0, setup_count = gsc_context::kSetupStreams;
    cudaEvent_t stage1_ev[gsc_context::kSetupStreams] = {};
    std::vector<uint32_t> small;     // indices of the instances the batched kernels run
    std::vector<BigInstance> big;    // the instances the one-problem kernels run
    WorkTotals tot{}, tot_all{};
    WorkList wl{}, wl_all{};
    uint32_t step_launches = 0;      // kernel launches of one iteration step
    BatchShape shape{};
    uint32_t wmax = 1;
    size_t smem = 0;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    BatchShape graph_shape{};
    gsc_batch_report t{};
    uint32_t last_launches = 0;
    ~gsc_batch() {
        release_batch_graph(this);
        probs.clear();
        abs.clear();
        device_release_all(ctx, pool, own, own_bytes);
        uint64_t tb = 0;
        for (auto& t : setup_tmp) device_release_all(ctx, pool, t, tb);
        pinned_put(ctx, pin_early, pin_early_bytes);
        pinned_put(ctx, pin_late, pin_late_bytes);
        for (auto e : stage1_ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace {

struct ShapeKey {
    uint32_t wmax, n, sat_log, words_log, nv;
    bool operator<(const ShapeKey& o) const {
        return std::tie(wmax, n, sat_log, words_log, nv) < std::tie(o.wmax, o.n, o.sat_log, o.words_log, o.nv);
    }
};
std::mutex g_tune_mu;
std::map<ShapeKey, BatchShape> g_tuned;

uint32_t log2_ceil(uint64_t v) {
    uint32_t l = 0;
    while ((1ull << l) < v && l < 63) ++l;
    return l;
}

// Work lists with `chunk` word positions per task: the small instances'
// (the batched kernels) and every instance's (init and status).
int upload_list(gsc_batch* b, uint32_t chunk) {
    std::vector<const gsc_problem*> probs;
    std::vector<uint32_t> slots;
    for (uint32_t i : b->small) {
        probs.push_back(b->probs[i].get());
        slots.push_back(i);
    }
    build_work_list(probs, slots, chunk, b->hlist, b->tot);
    probs.clear();
    slots.clear();
    for (uint32_t i = 0; i < b->probs.size(); ++i) {
        probs.push_back(b->probs[i].get());
        slots.push_back(i);
    }
    build_work_list(probs, slots, chunk, b->hlist_all, b->tot_all);
    // A new upload (autotuning) waits until the previous one has read the
    // pinned lists; the first does not wait.
    if (b->lists_uploaded) GSC_CU(b->ctx, cudaStreamSynchronize(b->ctx->stream));
    const size_t words = b->probs.size() + 4 * (b->probs.size() + 1);
    uint32_t* pin_small = b->hlist_pin;
    uint32_t* pin_all = b->hlist_pin + words;
    std::memcpy(pin_small, b->hlist.data(), b->hlist.size() * 4);
    std::memcpy(pin_all, b->hlist_all.data(), b->hlist_all.size() * 4);
    GSC_CU(b->ctx, cudaMemcpyAsync(b->dlist, pin_small, b->hlist.size() * 4, cudaMemcpyHostToDevice, b->ctx->stream));
    GSC_CU(b->ctx, cudaMemcpyAsync(b->dlist_all, pin_all, b->hlist_all.size() * 4, cudaMemcpyHostToDevice,
                                   b->ctx->stream));
    b->lists_uploaded = true;
    b->wl = device_work_list(b->dlist, static_cast<uint32_t>(b->small.size()), chunk, nullptr, b->drunning);
    b->wl_all = device_work_list(b->dlist_all, static_cast<uint32_t>(b->probs.size()), chunk, b->hfc_dev, b->drunning);
    return GSC_OK;
}

cudaError_t enqueue_step(gsc_batch* b, cudaGraphConditionalHandle cond, int use_cond, uint32_t* launches) {
    return launch_batch_step(b->ddesc, b->wl, b->tot, b->wl_all, b->big.data(), static_cast<uint32_t>(b->big.size()),
                             b->shape, b->wmax, b->smem, sm_count(b->ctx), cond, use_cond, b->ctx->stream, launches);
}

int enqueue_iterations(gsc_batch* b, uint32_t count, uint32_t* launches) {
    for (uint32_t i = 0; i < count; ++i) GSC_CU(b->ctx, enqueue_step(b, 0, 0, launches));
    return GSC_OK;
}

// Time the solve from a fresh start (up to kTuneIterations iterations,
// checked every kTuneChunk: the first iterations test every pair, the later
// ones only the pairs near states that left D', and the best shape differs
// between the two) under each candidate shape; keep the fastest.  Candidates: one task per block (64 / 128 / 256
// threads) and one task per warp (4 or 8 warps a block), each with one
// block per task or a persistent grid, and chunks of 256 or 1,024 words; a
// warp shape whose staging does not fit a block's shared memory is left out.
// A single trial of a few iterations varies by a few percent between runs,
// so the three fastest shapes are timed twice more and each keeps its best
// time.
int autotune(gsc_batch* b) {
    gsc_context* ctx = b->ctx;
    const int sms = sm_count(ctx);
    struct Trial {
        uint32_t threads, warp;
    };
    const Trial trials[] = {{64, 0}, {128, 0}, {256, 0}, {128, 1}, {256, 1}};
    const uint32_t per_sm[] = {0, 4, 8, 16};
    const uint32_t chunks[] = {256, 1024};
    constexpr uint32_t kTuneChunk = 8, kTuneIterations = 32;
    cudaEvent_t e0, e1;
    GSC_CU(ctx, cudaEventCreate(&e0));
    GSC_CU(ctx, cudaEventCreate(&e1));
    uint32_t listed = 0;   // chunk of the uploaded work lists
    auto time_shape = [&](const BatchShape& cand, float* ms) -> int {
        if (cand.chunk != listed) {
            GSC_TRY(upload_list(b, cand.chunk));
            listed = cand.chunk;
        }
        b->shape = cand;
        cudaError_t e = launch_batch_init(b->ddesc, b->wl, b->tot, sms, ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(e0, ctx->stream);
        for (uint32_t done = 0; e == cudaSuccess && done < kTuneIterations; done += kTuneChunk) {
            for (uint32_t r = 0; e == cudaSuccess && r < kTuneChunk; ++r)
                e = launch_batch_iteration(b->ddesc, b->wl, b->tot, b->shape, b->wmax, b->smem, sms, 0, 0,
                                           ctx->stream, nullptr);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b->hrunning, b->drunning, 4, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e == cudaSuccess && *b->hrunning == 0) break;
        }
        if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
        if (e != cudaSuccess) return fail(ctx, GSC_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
        return GSC_OK;
    };
    std::vector<std::pair<float, BatchShape>> timed;
    int status = GSC_OK;
    for (uint32_t ch : chunks) {
        for (const Trial& tr : trials) {
            for (uint32_t ps : per_sm) {
                const BatchShape cand{tr.threads, ps * static_cast<uint32_t>(sms), ch, tr.warp};
                if (batch_sat_smem(cand, b->smem) > kFusedSmemMax) continue;
                float ms = 0.f;
                status = time_shape(cand, &ms);
                if (status != GSC_OK) break;
                timed.emplace_back(ms, cand);
            }
            if (status != GSC_OK) break;
        }
        if (status != GSC_OK) break;
    }
    if (status == GSC_OK && timed.empty()) status = fail(ctx, GSC_ERR_UNSUPPORTED, "autotune: no shape fits");
    if (status == GSC_OK) {
        std::stable_sort(timed.begin(), timed.end(),
                         [](const std::pair<float, BatchShape>& x, const std::pair<float, BatchShape>& y) {
                             return x.first < y.first;
                         });
        timed.resize(std::min<size_t>(timed.size(), 3));
        for (int round = 0; round < 2 && status == GSC_OK; ++round)
            for (auto& t : timed) {
                float ms = 0.f;
                status = time_shape(t.second, &ms);
                if (status != GSC_OK) break;
                t.first = std::min(t.first, ms);
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status != GSC_OK) return status;
    const auto best = std::min_element(timed.begin(), timed.end(),
                                       [](const std::pair<float, BatchShape>& x,
                                          const std::pair<float, BatchShape>& y) { return x.first < y.first; });
    b->shape = best->second;
    return upload_list(b, b->shape.chunk);
}

void release_batch_graph(gsc_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

int build_batch_graph(gsc_batch* b) {
    gsc_context* ctx = b->ctx;
    cudaStream_t st = ctx->stream;
    release_batch_graph(b);
    const int sms = sm_count(ctx);
    cudaGraph_t g = nullptr, ginit = nullptr;
    GSC_CU(ctx, cudaGraphCreate(&g, 0));
    b->graph = g;
    GSC_CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = launch_batch_init(b->ddesc, b->wl_all, b->tot_all, sms, st);
    cudaError_t e2 = cudaStreamEndCapture(st, &ginit);
    GSC_CU(ctx, e);
    GSC_CU(ctx, e2);
    cudaGraphNode_t init_node;
    e = cudaGraphAddChildGraphNode(&init_node, g, nullptr, 0, ginit);
    cudaGraphDestroy(ginit);
    GSC_CU(ctx, e);
    cudaGraphConditionalHandle handle;
    GSC_CU(ctx, cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    GSC_CU(ctx, cudaGraphAddNode(&cnode, g, &init_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    GSC_CU(ctx, cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    e = enqueue_step(b, handle, 1, nullptr);
    cudaGraph_t body_out = nullptr;
    e2 = cudaStreamEndCapture(st, &body_out);
    GSC_CU(ctx, e);
    GSC_CU(ctx, e2);
    GSC_CU(ctx, cudaGraphInstantiate(&b->exec, g, 0));
    b->graph_shape = b->shape;
    return GSC_OK;
}

// Carves `bytes` (rounded up to 16) off the front of a pinned block.
char* carve16(char*& p, size_t bytes) {
    char* r = p;
    p += (bytes + 15) & ~size_t(15);
    return r;
}

// The context's set-up streams for one batch (instance i on stream
// base + i % count), so that the small set-up kernels of different
// instances run side by side.  They have the device's highest stream
// priority: in a pipelined run their blocks go ahead of a solve that fills
// the GPU.  They are created once per context; a batch that fails drains
// the streams it used before its memory is released, a batch that succeeds
// only joins them into the context stream (no host wait).  The two set-up
// phases of a batch (batch_begin, batch_finish) each hold one of these over
// the same streams.
struct SetupStreams {
    static constexpr int kSetupStreams = gsc_context::kSetupStreams;
    gsc_context* ctx = nullptr;
    uint32_t base = 0, count = kSetupStreams;
    bool ok = false;
    ~SetupStreams() {
        if (ok || !ctx) return;
        for (uint32_t k = 0; k < count; ++k)
            if (ctx->setup[base + k]) cudaStreamSynchronize(ctx->setup[base + k]);
    }
    void attach(gsc_context* c, uint32_t b0, uint32_t n) {
        ctx = c;
        base = b0;
        count = n;
    }
    // Creates the context's streams at first use; the streams in use start
    // after the work queued on `after` so far.
    cudaError_t create(gsc_context* c, cudaStream_t after, uint32_t b0, uint32_t n) {
        attach(c, b0, n);
        cudaError_t r = cudaSuccess;
        if (!ctx->setup[0]) {
            int least = 0, greatest = 0;
            r = cudaDeviceGetStreamPriorityRange(&least, &greatest);
            for (auto& x : ctx->setup)
                if (r == cudaSuccess) r = cudaStreamCreateWithPriority(&x, cudaStreamNonBlocking, greatest);
            for (auto& e : ctx->setup_ev)
                if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            if (r != cudaSuccess) return r;
        }
        r = cudaEventRecord(ctx->setup_ev[kSetupStreams], after);
        for (uint32_t k = 0; k < count; ++k)
            if (r == cudaSuccess) r = cudaStreamWaitEvent(ctx->setup[base + k], ctx->setup_ev[kSetupStreams], 0);
        return r;
    }
    cudaStream_t of(uint32_t i) const { return ctx->setup[base + i % count]; }
    // evs[k] marks what stream base + k has queued so far.
    cudaError_t mark(cudaEvent_t* evs) {
        for (uint32_t k = 0; k < count; ++k) {
            cudaError_t r = cudaSuccess;
            if (!evs[k]) r = cudaEventCreateWithFlags(&evs[k], cudaEventDisableTiming);
            if (r == cudaSuccess) r = cudaEventRecord(evs[k], ctx->setup[base + k]);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
    // Host wait for the marks (later work on the streams is not waited for).
    cudaError_t wait(cudaEvent_t* evs) {
        for (uint32_t k = 0; k < count; ++k) {
            const cudaError_t r = cudaEventSynchronize(evs[k]);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
    // `st` waits for everything enqueued on the streams in use.
    cudaError_t join(cudaStream_t st) {
        for (uint32_t k = 0; k < count; ++k) {
            cudaError_t r = cudaEventRecord(ctx->setup_ev[base + k], ctx->setup[base + k]);
            if (r == cudaSuccess) r = cudaStreamWaitEvent(st, ctx->setup_ev[base + k], 0);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
};

// Set-up phase 1: stage 1 of every instance (abstraction tables, masks,
// boxes, x classes, representatives, plan records) queued on set-up streams
// base..base+streams-1, with no host wait.
int batch_begin(gsc_batch* b, uint32_t count, const gsc_model_desc* models, const gsc_query_desc* queries,
                uint32_t base, uint32_t streams) {
    gsc_context* ctx = b->ctx;
    b->pool = ctx->pool.get();
    b->setup_base = base;
    b->setup_count = streams;
    SetupStreams ss;
    GSC_CU(ctx, ss.create(ctx, ctx->stream, base, streams));
    // Pinned host memory in two carved blocks from the context's cache.
    {
        const size_t bytes = ((sizeof(PlanRecord) * count + 15) & ~size_t(15)) + 16 +
                             ((sizeof(FixControl) * count + 15) & ~size_t(15));
        GSC_CU(ctx, pinned_get(ctx, bytes, &b->pin_early, &b->pin_early_bytes));
        char* q = static_cast<char*>(b->pin_early);
        b->hplans = reinterpret_cast<PlanRecord*>(carve16(q, sizeof(PlanRecord) * count));
        b->hrunning = reinterpret_cast<uint32_t*>(carve16(q, sizeof(uint32_t)));
        b->hfc = reinterpret_cast<FixControl*>(carve16(q, sizeof(FixControl) * count));
        std::memset(b->pin_early, 0, bytes);
        char* dq = nullptr;
        GSC_CU(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&dq), b->pin_early, 0));
        b->hplans_dev = reinterpret_cast<PlanRecord*>(dq + (reinterpret_cast<char*>(b->hplans) -
                                                             static_cast<char*>(b->pin_early)));
        b->hfc_dev = reinterpret_cast<FixControl*>(dq + (reinterpret_cast<char*>(b->hfc) -
                                                          static_cast<char*>(b->pin_early)));
    }
    b->setup_tmp.assign(count, {});
    for (uint32_t i = 0; i < count; ++i) {
        std::unique_ptr<gsc_abstraction> a(new (std::nothrow) gsc_abstraction());
        if (!a) return GSC_ERR_OUT_OF_MEMORY;
        a->ctx = ctx;
        a->model = models[i];
        a->pool = b->pool;
        std::string err;
        const int s = grid_from_model(&models[i], &a->g, &err);
        if (s != GSC_OK) return fail(ctx, s, "instance " + std::to_string(i) + ": " + err);
        if (a->g.rows * a->g.W >= 0xFFFFFFFFull)
            return fail(ctx, GSC_ERR_UNSUPPORTED, "instance " + std::to_string(i) + ": grid too large for a batch");
        GSC_TRY(abstraction_enqueue(a.get(), ss.of(i), b->setup_tmp[i]));
        b->abs.push_back(std::move(a));
    }
    for (uint32_t i = 0; i < count; ++i) {
        std::unique_ptr<gsc_problem> p(new (std::nothrow) gsc_problem());
        if (!p) return GSC_ERR_OUT_OF_MEMORY;
        p->ctx = ctx;
        p->abs = b->abs[i].get();
        p->g = b->abs[i]->g;
        p->pool = b->pool;
        p->stream = ss.of(i);
        p->method = GSC_METHOD_FUSED;
        p->hplan = b->hplans + i;
        p->hplan_dev = b->hplans_dev + i;
        const int s = problem_stage1(p.get(), &queries[i]);
        if (s != GSC_OK) return fail(ctx, s, "instance " + std::to_string(i) + ": " + ctx->last_error);
        b->probs.push_back(std::move(p));
    }
    GSC_CU(ctx, ss.mark(b->stage1_ev));
    ss.ok = true;
    return GSC_OK;
}

// Set-up phase 2: one host wait for the stage-1 work of batch_begin (the
// plan records), then stage 2 of every instance, the instance table, work
// lists and launch shapes (autotuned on request).
int batch_finish(gsc_batch* b, const gsc_batch_options* opt) {
    gsc_context* ctx = b->ctx;
    cudaStream_t st = ctx->stream;
    const uint32_t count = static_cast<uint32_t>(b->probs.size());
    SetupStreams ss;
    ss.attach(ctx, b->setup_base, b->setup_count);
    GSC_CU(ctx, ss.wait(b->stage1_ev));
    for (auto& t : b->setup_tmp) {
        uint64_t tb = 0;
        device_release_all(ctx, b->pool, t, tb);
    }
    b->setup_tmp.clear();
    for (uint32_t i = 0; i < count; ++i) {
        gsc_problem* p = b->probs[i].get();
        int s = problem_plan(p);
        if (s == GSC_OK) s = problem_stage2(p);
        if (s != GSC_OK) return fail(ctx, s, "instance " + std::to_string(i) + ": " + ctx->last_error);
    }
    // Later work on the context stream (init, solves, reads) follows the set-up.
    GSC_CU(ctx, ss.join(st));
    ss.ok = true;
    for (auto& p : b->probs) p->stream = st;
    // Pinned staging of the per-iteration counters for reads.
    uint64_t stats_words = 0;
    for (uint32_t i = 0; i < count; ++i) {
        b->stats_off.push_back(stats_words);
        stats_words += static_cast<uint64_t>(kStatsCols) * b->probs[i]->stats_cap;
    }
    const size_t list_bytes = 2 * 4ull * (count + 4ull * (count + 1));
    {
        const size_t bytes = ((sizeof(unsigned long long) * stats_words + 15) & ~size_t(15)) +
                             ((sizeof(InstanceDesc) * count + 15) & ~size_t(15)) + ((list_bytes + 15) & ~size_t(15));
        GSC_CU(ctx, pinned_get(ctx, bytes, &b->pin_late, &b->pin_late_bytes));
        char* q = static_cast<char*>(b->pin_late);
        b->hstats = reinterpret_cast<unsigned long long*>(carve16(q, sizeof(unsigned long long) * stats_words));
        b->hdesc_pin = reinterpret_cast<InstanceDesc*>(carve16(q, sizeof(InstanceDesc) * count));
        b->hlist_pin = reinterpret_cast<uint32_t*>(carve16(q, list_bytes));
    }
    // Instance table, work lists and launch shapes; wmax and the shared
    // memory of the batched satisfaction kernel come from the small instances.
    std::vector<InstanceDesc> hd(count);
    uint32_t wmax = 1, nv_any = 0;
    size_t smem = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const gsc_problem* p = b->probs[i].get();
        hd[i] = make_instance(p);
        if (instance_smem(p) > kFusedSmemMax)
            return fail(ctx, GSC_ERR_UNSUPPORTED, "instance " + std::to_string(i) + ": needs too much shared memory");
        if (is_big_instance(p->g)) {
            b->big.push_back(BigInstance{p->g, hd[i].a});
            continue;
        }
        b->small.push_back(i);
        wmax = std::max(wmax, p->g.W);
        smem = std::max(smem, instance_smem(p));
        nv_any |= p->need_valid ? 1u : 0u;
    }
    b->wmax = wmax_of(wmax);
    b->smem = smem;
    b->step_launches = 3 * static_cast<uint32_t>(b->big.size()) + (b->small.empty() ? 0u : 3u) + 1u;
    void* q = nullptr;
    GSC_TRY(device_alloc(ctx, b->pool, b->own, b->own_bytes, &q, sizeof(InstanceDesc) * count));
    b->ddesc = static_cast<InstanceDesc*>(q);
    GSC_TRY(device_alloc(ctx, b->pool, b->own, b->own_bytes, &q, 4ull * (count + 4ull * (count + 1))));
    b->dlist = static_cast<uint32_t*>(q);
    GSC_TRY(device_alloc(ctx, b->pool, b->own, b->own_bytes, &q, 4ull * (count + 4ull * (count + 1))));
    b->dlist_all = static_cast<uint32_t*>(q);
    GSC_TRY(device_alloc(ctx, b->pool, b->own, b->own_bytes, &q, 4));
    b->drunning = static_cast<uint32_t*>(q);
    std::memcpy(b->hdesc_pin, hd.data(), sizeof(InstanceDesc) * count);
    GSC_CU(ctx, cudaMemcpyAsync(b->ddesc, b->hdesc_pin, sizeof(InstanceDesc) * count, cudaMemcpyHostToDevice, st));

    const int sms = sm_count(ctx);
    b->shape.sat_threads = (opt && opt->sat_threads) ? opt->sat_threads : 128;
    b->shape.sat_blocks = (opt ? opt->sat_blocks_per_sm : 0) * static_cast<uint32_t>(sms);
    b->shape.chunk = (opt && opt->chunk_words) ? opt->chunk_words : 2048;
    b->shape.warp = (opt && opt->sat_warp_tasks) ? 1u : 0u;
    if (b->shape.sat_threads != 64 && b->shape.sat_threads != 128 && b->shape.sat_threads != 256)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "sat_threads must be 64, 128 or 256");
    if (b->shape.chunk < 256 || b->shape.chunk % 256)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "chunk_words must be a positive multiple of 256");
    if (batch_sat_smem(b->shape, smem) > kFusedSmemMax)
        return fail(ctx, GSC_ERR_UNSUPPORTED, "batch: one task per warp needs more shared memory than a block has");
    GSC_TRY(upload_list(b, b->shape.chunk));
    b->t.tuned = 0;
    if (opt && opt->autotune && !b->small.empty()) {
        uint64_t words = 0;
        for (uint32_t i : b->small) words += hd[i].words;
        const ShapeKey key{b->wmax, static_cast<uint32_t>(b->small.size()), log2_ceil(b->tot.sat), log2_ceil(words),
                           nv_any};
        bool hit = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tuned.find(key);
            if (it != g_tuned.end()) {
                b->shape = it->second;
                hit = true;
            }
        }
        if (hit) {
            GSC_TRY(upload_list(b, b->shape.chunk));
            b->t.tuned = 2;
        } else {
            const auto t0 = std::chrono::steady_clock::now();
            GSC_TRY(autotune(b));
            b->t.tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            b->t.tuned = 1;
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tuned[key] = b->shape;
        }
    }
    b->t.instances = count;
    return GSC_OK;
}

int batch_create(gsc_batch* b, uint32_t count, const gsc_model_desc* models, const gsc_query_desc* queries,
                 const gsc_batch_options* opt) {
    GSC_TRY(batch_begin(b, count, models, queries, 0, gsc_context::kSetupStreams));
    return batch_finish(b, opt);
}

// Queues the copies of every instance's results on `st` (which must follow
// the solve and the unpacking of the reachable sets): valid, candidate and
// reachable masks, controller, reach_step, and rows[i] + 1 rows of
// per-iteration counters into the pinned staging.
int read_enqueue(gsc_batch* b, const gsc_result* out, cudaStream_t st, const std::vector<uint32_t>& rows) {
    gsc_context* ctx = b->ctx;
    for (size_t i = 0; i < b->probs.size(); ++i) {
        gsc_problem* p = b->probs[i].get();
        const GridInfo& g = p->g;
        const gsc_result* r = out + i;
        if (r->valid_mask) GSC_CU(ctx, cudaMemcpyAsync(r->valid_mask, p->valid, g.S, cudaMemcpyDeviceToHost, st));
        if (r->candidate_mask)
            GSC_CU(ctx, cudaMemcpyAsync(r->candidate_mask, p->cand, g.S, cudaMemcpyDeviceToHost, st));
        if (r->reachable_mask)
            GSC_CU(ctx, cudaMemcpyAsync(r->reachable_mask, p->reach8, g.S, cudaMemcpyDeviceToHost, st));
        if (r->controller)
            GSC_CU(ctx, cudaMemcpyAsync(r->controller, p->controller, g.S * 4, cudaMemcpyDeviceToHost, st));
        if (r->reach_step)
            GSC_CU(ctx, cudaMemcpyAsync(r->reach_step, p->reach_step, g.S * 4, cudaMemcpyDeviceToHost, st));
        if (rows[i] && (r->iter_new_reachable || r->iter_new_certified))
            GSC_CU(ctx, cudaMemcpyAsync(b->hstats + b->stats_off[i], p->stats,
                                        sizeof(unsigned long long) * kStatsCols * (rows[i] + 1),
                                        cudaMemcpyDeviceToHost, st));
    }
    return GSC_OK;
}

// Counter rows of instance i that a read returns: the iterations run, at most
// the caller's capacity and the staged rows.
uint32_t read_rows(const gsc_batch* b, const gsc_result* r, size_t i) {
    return std::min<uint32_t>({b->hfc[i].iter, r->iter_capacity, b->probs[i]->stats_cap - 1});
}

// Once the solve has finished: the result fields from the control records
// (the status kernel stores them in pinned memory after every iteration)
// and, once the copies of read_enqueue have finished, the per-iteration
// counters.
void read_finish(gsc_batch* b, gsc_result* out) {
    for (size_t i = 0; i < b->probs.size(); ++i) {
        const gsc_problem* p = b->probs[i].get();
        const GridInfo& g = p->g;
        const FixControl& fc = b->hfc[i];
        gsc_result* r = out + i;
        for (int d = 0; d < 4; ++d) r->shape[d] = g.n[d];
        r->input_shape[0] = g.ma;
        r->input_shape[1] = g.mw;
        r->states = g.S;
        r->inputs = g.M;
        r->pairs = g.S * g.M;
        r->iterations = fc.iter;
        r->converged = static_cast<int32_t>(fc.converged);
        r->message = static_cast<int32_t>(fc.message ? fc.message : GSC_MSG_MAX_ITERATIONS);
        r->certified_candidates = fc.certified;
        r->reachable_states = fc.reachable;
        r->candidate_count = fc.candidate_count;
        r->valid_count = fc.valid_count;
        const unsigned long long* hs = b->hstats + b->stats_off[i];
        const uint32_t rows = read_rows(b, r, i);
        for (uint32_t k = 0; k < rows; ++k) {
            if (r->iter_new_reachable) r->iter_new_reachable[k] = hs[kStatsCols * (k + 1)];
            if (r->iter_new_certified) r->iter_new_certified[k] = hs[kStatsCols * (k + 1) + 1];
        }
    }
}

}  // namespace

extern "C" {

int gsc_batch_create(gsc_context* ctx, uint32_t count, const gsc_model_desc* models, const gsc_query_desc* queries,
                     const gsc_batch_options* options, gsc_batch** out) {
    if (!ctx || !models || !queries || !out || count == 0) return GSC_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cudaGetLastError();
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<gsc_batch> b(new (std::nothrow) gsc_batch());
    if (!b) return GSC_ERR_OUT_OF_MEMORY;
    b->ctx = ctx;
    const int s = batch_create(b.get(), count, models, queries, options);
    if (s != GSC_OK) {
        cudaStreamSynchronize(ctx->stream);   // nothing of the failed batch may still be in flight
        return s;
    }
    b->t.create_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out = b.release();
    return GSC_OK;
}

int gsc_batch_solve(gsc_batch* b, uint32_t flags) {
    if (!b) return GSC_ERR_INVALID_ARGUMENT;
    gsc_context* ctx = b->ctx;
    cudaGetLastError();
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int sms = sm_count(ctx);
    GSC_CU(ctx, cudaEventRecord(ctx->ev[0], st));
    uint32_t launches = 0;
    if (flags & GSC_SOLVE_GRAPH) {
        if (!b->exec || std::memcmp(&b->graph_shape, &b->shape, sizeof(BatchShape)) != 0)
            GSC_TRY(build_batch_graph(b));
        GSC_CU(ctx, cudaGraphLaunch(b->exec, st));
        launches = 0;   // counted below from the iterations run
    } else {
        GSC_CU(ctx, launch_batch_init(b->ddesc, b->wl_all, b->tot_all, sms, st));
        launches = 1;
        uint32_t cap = 0;
        for (const auto& p : b->probs) cap = std::max(cap, p->stats_cap);
        uint32_t done = 0, chunk = 4;
        while (true) {
            GSC_TRY(enqueue_iterations(b, chunk, &launches));
            done += chunk;
            GSC_CU(ctx, cudaMemcpyAsync(b->hrunning, b->drunning, 4, cudaMemcpyDeviceToHost, st));
            GSC_CU(ctx, cudaStreamSynchronize(st));
            if (*b->hrunning == 0) break;
            if (done > cap + 64) return fail(ctx, GSC_ERR_TIMEOUT, "batch fixpoint did not stop within its bound");
            if (chunk < 32) chunk *= 2;
        }
    }
    GSC_CU(ctx, cudaEventRecord(ctx->ev[1], st));
    GSC_CU(ctx, cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    GSC_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    b->t.solve_ms = ms;
    b->last_launches = (flags & GSC_SOLVE_GRAPH) ? 0xFFFFFFFFu : launches;
    b->t.max_iterations_run = 0;
    b->t.pair_tests = 0;
    return GSC_OK;
}

int gsc_batch_read(gsc_batch* b, uint32_t index, gsc_result* out) {
    if (!b || !out || index >= b->probs.size()) return GSC_ERR_INVALID_ARGUMENT;
    return gsc_problem_read(b->probs[index].get(), out);
}

int gsc_batch_timings(gsc_batch* b, gsc_batch_report* out) {
    if (!b || !out) return GSC_ERR_INVALID_ARGUMENT;
    gsc_context* ctx = b->ctx;
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    // Per-instance iteration counts and pair tests of the last solve.
    uint32_t maxit = 0;
    uint64_t tests = 0;
    for (const auto& p : b->probs) {
        FixControl fc;
        GSC_CU(ctx, cudaMemcpyAsync(&fc, p->fc, sizeof(fc), cudaMemcpyDeviceToHost, ctx->stream));
        GSC_CU(ctx, cudaStreamSynchronize(ctx->stream));
        const uint32_t iters = std::min<uint32_t>(fc.iter, p->stats_cap - 1);
        maxit = std::max(maxit, iters);
        if (iters) {
            std::vector<unsigned long long> hs(static_cast<size_t>(kStatsCols) * (iters + 1));
            GSC_CU(ctx, cudaMemcpyAsync(hs.data(), p->stats, hs.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
            GSC_CU(ctx, cudaStreamSynchronize(ctx->stream));
            for (uint32_t i = 1; i <= iters; ++i) tests += hs[kStatsCols * i + 2];
        }
    }
    b->t.max_iterations_run = maxit;
    b->t.pair_tests = tests;
    // Graph solves run the body once per iteration of the longest instance.
    b->t.kernel_launches =
        b->last_launches == 0xFFFFFFFFu ? 1 + b->step_launches * std::max<uint32_t>(maxit, 1) : b->last_launches;
    b->t.sat_threads = b->shape.sat_threads;
    const int sms = sm_count(ctx);
    b->t.sat_blocks_per_sm = b->shape.sat_blocks / static_cast<uint32_t>(sms);
    b->t.chunk_words = b->shape.chunk;
    b->t.sat_warp_tasks = b->shape.warp;
    uint64_t held = b->own_bytes;
    for (const auto& a : b->abs) held += a->bytes;
    for (const auto& p : b->probs) held += p->bytes;
    b->t.device_bytes = held;
    *out = b->t;
    return GSC_OK;
}

// Streams of a pipelined run.  Every exit drains them, the context stream
// and the set-up streams before the parts' memory is released.
struct RunStreams {
    gsc_context* ctx = nullptr;
    cudaStream_t solve[2] = {nullptr, nullptr}, copy = nullptr;
    cudaEvent_t ready = nullptr;
    std::vector<cudaEvent_t> solved;
    ~RunStreams() {
        for (auto s : {solve[0], solve[1], copy})
            if (s) {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
        if (ctx) {
            cudaStreamSynchronize(ctx->stream);
            for (auto s : ctx->setup)
                if (s) cudaStreamSynchronize(s);
        }
        if (ready) cudaEventDestroy(ready);
        for (auto e : solved) cudaEventDestroy(e);
    }
};

int gsc_batch_run(gsc_context* ctx, uint32_t count, const gsc_model_desc* models, const gsc_query_desc* queries,
                  const gsc_batch_options* options, uint32_t part_instances, gsc_result* results) {
    if (!ctx || !models || !queries || !results || count == 0) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    const uint32_t part = part_instances ? part_instances : std::max<uint32_t>(1, (count + 7) / 8);
    const uint32_t nparts = (count + part - 1) / part;
    const int sms = sm_count(ctx);
    std::vector<std::unique_ptr<gsc_batch>> parts;   // destroyed after `rs` drained the streams
    RunStreams rs;
    rs.ctx = ctx;
    for (auto& x : rs.solve) GSC_CU(ctx, cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    GSC_CU(ctx, cudaStreamCreateWithFlags(&rs.copy, cudaStreamNonBlocking));
    GSC_CU(ctx, cudaEventCreateWithFlags(&rs.ready, cudaEventDisableTiming));
    gsc_batch_options opt = options ? *options : gsc_batch_options{};
    auto range = [&](uint32_t k) {
        const uint32_t f = k * part, n = std::min(part, count - f);
        return "instances " + std::to_string(f) + ".." + std::to_string(f + n - 1) + ": ";
    };
    // Stage 1 of part k, queued on half of the set-up streams (even parts
    // the first half, odd parts the second), so that the next part's stage 1
    // and this part's stage 2 do not queue behind each other.
    auto begin_part = [&](uint32_t k) -> int {
        const uint32_t f = k * part, n = std::min(part, count - f);
        std::unique_ptr<gsc_batch> b(new (std::nothrow) gsc_batch());
        if (!b) return GSC_ERR_OUT_OF_MEMORY;
        b->ctx = ctx;
        parts.push_back(std::move(b));
        const uint32_t half = gsc_context::kSetupStreams / 2;
        const int s = batch_begin(parts.back().get(), n, models + f, queries + f, (k & 1) * half, half);
        return s == GSC_OK ? GSC_OK : fail(ctx, s, range(k) + ctx->last_error);
    };
    GSC_TRY(begin_part(0));
    for (uint32_t k = 0; k < nparts; ++k) {
        const uint32_t f = k * part, n = std::min(part, count - f);
        // The next part's stage 1 is queued before this part's plan wait,
        // except while this part tunes the launch shapes (its trials run alone).
        const bool tunes = k == 0 && opt.autotune;
        if (!tunes && k + 1 < nparts) GSC_TRY(begin_part(k + 1));
        gsc_batch* b = parts[k].get();
        int s = batch_finish(b, &opt);
        if (s == GSC_OK && !b->exec) s = build_batch_graph(b);
        if (s != GSC_OK) return fail(ctx, s, range(k) + ctx->last_error);
        if (tunes) {
            // Later parts take the first part's shapes: no trials beside a solve.
            opt.autotune = 0;
            opt.sat_threads = b->shape.sat_threads;
            opt.sat_blocks_per_sm = b->shape.sat_blocks / static_cast<uint32_t>(sms);
            opt.chunk_words = b->shape.chunk;
            opt.sat_warp_tasks = b->shape.warp;
            if (k + 1 < nparts) GSC_TRY(begin_part(k + 1));
        }
        // The solve follows the part's set-up (joined into the context
        // stream).  Parts alternate between two solve streams, so that a
        // part's last iterations, which few instances still run, share the
        // GPU with the next part's solve.
        cudaStream_t solve = rs.solve[k & 1];
        GSC_CU(ctx, cudaEventRecord(rs.ready, ctx->stream));
        GSC_CU(ctx, cudaStreamWaitEvent(solve, rs.ready, 0));
        GSC_CU(ctx, cudaGraphLaunch(b->exec, solve));
        // Unpack the reachable sets on the solve stream too, so the copy
        // stream carries copies only (its kernels would wait for SMs behind
        // the next part's solve).
        for (uint32_t i = 0; i < n; ++i) {
            gsc_problem* p = b->probs[i].get();
            if (results[f + i].reachable_mask)
                GSC_CU(ctx, launch_unpack_reach(p->g, p->fc, p->reach0, p->reach1, p->reach8, solve));
        }
        cudaEvent_t ev = nullptr;
        GSC_CU(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        rs.solved.push_back(ev);
        GSC_CU(ctx, cudaEventRecord(ev, solve));
        // The part's copies follow its solve with no host wait: the
        // iteration counts are not known yet, so every counter row a result
        // can take is staged.
        std::vector<uint32_t> rows(n);
        for (uint32_t i = 0; i < n; ++i)
            rows[i] = std::min<uint32_t>(results[f + i].iter_capacity, b->probs[i]->stats_cap - 1);
        GSC_CU(ctx, cudaStreamWaitEvent(rs.copy, ev, 0));
        GSC_TRY(read_enqueue(b, results + f, rs.copy, rows));
    }
    // While the last copies run, each part's graph goes as soon as its solve
    // has finished (destroying a graph costs the host about as much as
    // building it).
    for (uint32_t k = 0; k < nparts; ++k) {
        GSC_CU(ctx, cudaEventSynchronize(rs.solved[k]));
        release_batch_graph(parts[k].get());
    }
    GSC_CU(ctx, cudaStreamSynchronize(rs.copy));
    for (uint32_t k = 0; k < nparts; ++k) read_finish(parts[k].get(), results + k * part);
    return GSC_OK;
}

int gsc_batch_read_all(gsc_batch* b, gsc_result* out) {
    if (!b || !out) return GSC_ERR_INVALID_ARGUMENT;
    gsc_context* ctx = b->ctx;
    cudaGetLastError();
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    // One host wait for the solve: the control records are then final and
    // give each reachable set's buffer and counter rows.
    GSC_CU(ctx, cudaStreamSynchronize(st));
    std::vector<uint32_t> rows(b->probs.size());
    for (size_t i = 0; i < b->probs.size(); ++i) {
        gsc_problem* p = b->probs[i].get();
        if (out[i].reachable_mask)
            GSC_CU(ctx, launch_unpack_bits(p->g, (b->hfc[i].iter & 1) ? p->reach1 : p->reach0, p->reach8, st));
        rows[i] = read_rows(b, out + i, i);
    }
    GSC_TRY(read_enqueue(b, out, st, rows));
    GSC_CU(ctx, cudaStreamSynchronize(st));
    read_finish(b, out);
    return GSC_OK;
}

void gsc_batch_destroy(gsc_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
}

}  // extern "C"
