// gsc_server.cu -- the serving loop (gsc_server_* of include/gsc_b200.h).
//
// No counterpart in the reference.  One loop thread owns three streams:
//   prep   set-up of admitted queries (problem stage 1, plan, stage 2, init);
//   main   batched fixpoint steps over every running query (the kernels of
//          gsc_batch_kernels.cu on a task list of the running slots; a
//          query that fills the GPU alone runs the one-problem kernels in
//          the same step);
//   copy   results of stopped queries to the callers' buffers.
// A query moves QUEUED -> PREP1 -> PREP2 -> RUN -> COPY -> DONE.  Admission
// is in arrival order while a slot is free and the query's buffers fit the
// device pool (a fixed region of the budget); while a step runs, the loop
// keeps admitting and preparing, so set-up overlaps the iterations and new
// queries join the running set at the next step.  Each query keeps its own
// control record and tables, so its result does not depend on what else is
// running.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gsc_internal.hpp"

using namespace gsc_b200;
using namespace gsc_api;

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { kQueued, kPrep1, kPrep2, kRun, kCopy, kDone };

struct Req {
    uint64_t ticket = 0;
    const gsc_abstraction* abs = nullptr;
    gsc_query_desc q{};
    gsc_result* out = nullptr;
    std::unique_ptr<gsc_problem> p;
    ReqState state = kQueued;
    int status = GSC_OK;
    uint32_t slot = 0;
    cudaEvent_t ev = nullptr;
    FixControl fc{};
    Clock::time_point t_submit, t_done;
};

constexpr uint32_t kStatsRows = 4096;   // per-slot pinned staging of per-iteration counters

}  // namespace

struct gsc_server {
    gsc_context* ctx = nullptr;      // the caller's context (device, budget accounting)
    gsc_context ictx;                // the loop thread's own error slot and stream
    gsc_server_options opt{};
    std::unique_ptr<DevicePool> pool;
    cudaStream_t s_main = nullptr, s_prep = nullptr, s_copy = nullptr;
    cudaEvent_t ev_step = nullptr;
    // device
    InstanceDesc* ddesc = nullptr;
    uint32_t* dlist = nullptr;         // every running query: status
    uint32_t* dlist_small = nullptr;   // the running queries the batched kernels run
    void* dmem = nullptr;
    // pinned host
    InstanceDesc* hdesc = nullptr;
    uint32_t* hlist = nullptr;   // both lists, the small one after the other
    FixControl* hstatus = nullptr;       // pinned; the status kernel stores each step's records here
    FixControl* hstatus_dev = nullptr;   // its device address
    PlanRecord* hplans = nullptr;
    PlanRecord* hplans_dev = nullptr;   // their device address (stored by a kernel, not copied)
    unsigned long long* hstats = nullptr;   // [slot][kStatsRows][kStatsCols]
    // loop-thread state
    std::vector<uint32_t> free_slots;
    std::vector<Req*> prep1, prep2, running, copying;
    BatchShape shape{};
    uint64_t mem_epoch = 0;       // releases so far
    uint64_t blocked_epoch = ~0ull;   // mem_epoch when the head of the queue last did not fit
    // shared
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
    uint64_t next_ticket = 1;
    bool stopping = false;
    gsc_server_report st{};
    std::thread th;
    ~gsc_server();
};

namespace {

void finish(gsc_server* s, Req* r, int status) {
    r->t_done = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    r->status = status;
    r->state = kDone;
    s->st.completed++;
    if (status != GSC_OK) s->st.failed++;
    s->st.in_flight--;
    s->cv_done.notify_all();
}

void release(gsc_server* s, Req* r) {
    r->p.reset();
    s->mem_epoch++;
    s->free_slots.push_back(r->slot);
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.device_bytes_in_use = s->pool->used();
}

bool nothing_in_flight(const gsc_server* s) {
    return s->prep1.empty() && s->prep2.empty() && s->running.empty() && s->copying.empty();
}

// QUEUED -> PREP1 while a slot is free and stage 1 fits the pool.
bool admit(gsc_server* s) {
    bool any = false;
    // After the head of the queue did not fit, wait until memory is released.
    if (s->blocked_epoch == s->mem_epoch) return false;
    while (!s->free_slots.empty()) {
        Req* r = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->queue.empty()) break;
            r = s->queue.front();
            s->queue.pop_front();
            s->st.queued--;
        }
        r->slot = s->free_slots.back();
        s->free_slots.pop_back();
        r->p.reset(new (std::nothrow) gsc_problem());
        if (!r->p) {
            s->free_slots.push_back(r->slot);
            finish(s, r, GSC_ERR_OUT_OF_MEMORY);
            continue;
        }
        gsc_problem* p = r->p.get();
        p->ctx = &s->ictx;
        p->abs = r->abs;
        p->g = r->abs->g;
        p->pool = s->pool.get();
        p->stream = s->s_prep;
        p->method = GSC_METHOD_FUSED;
        p->hplan = s->hplans + r->slot;
        p->hplan_dev = s->hplans_dev + r->slot;
        int status = problem_stage1(p, &r->q);
        if (status == GSC_OK && cudaEventRecord(r->ev, s->s_prep) != cudaSuccess) status = GSC_ERR_CUDA;
        if (status == GSC_ERR_OUT_OF_MEMORY && !nothing_in_flight(s)) {
            // Wait for memory: back to the head of the queue.
            cudaStreamSynchronize(s->s_prep);   // stage-1 work already issued reads nothing freed below
            release(s, r);
            s->blocked_epoch = s->mem_epoch;
            std::lock_guard<std::mutex> lk(s->mu);
            s->queue.push_front(r);
            s->st.queued++;
            break;
        }
        if (status != GSC_OK) {
            cudaStreamSynchronize(s->s_prep);
            release(s, r);
            finish(s, r, status);
            continue;
        }
        r->state = kPrep1;
        s->prep1.push_back(r);
        any = true;
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.device_bytes_in_use = s->pool->used();
        s->st.peak_device_bytes = std::max(s->st.peak_device_bytes, s->st.device_bytes_in_use);
    }
    return any;
}

// PREP1 -> PREP2: plan, stage 2, instance record and init on the prep stream.
bool advance_prep1(gsc_server* s) {
    bool any = false;
    for (size_t i = 0; i < s->prep1.size();) {
        Req* r = s->prep1[i];
        const cudaError_t q = cudaEventQuery(r->ev);
        if (q == cudaErrorNotReady) {
            ++i;
            continue;
        }
        s->prep1.erase(s->prep1.begin() + i);
        any = true;
        gsc_problem* p = r->p.get();
        int status = q == cudaSuccess ? problem_plan(p) : GSC_ERR_CUDA;
        if (status == GSC_OK) status = problem_stage2(p);
        if (status == GSC_ERR_OUT_OF_MEMORY && !nothing_in_flight(s)) {
            cudaStreamSynchronize(s->s_prep);
            release(s, r);
            s->blocked_epoch = s->mem_epoch;
            std::lock_guard<std::mutex> lk(s->mu);
            s->queue.push_front(r);
            s->st.queued++;
            r->state = kQueued;
            continue;
        }
        if (status == GSC_OK) {
            s->hdesc[r->slot] = make_instance(p);
            cudaError_t e = cudaMemcpyAsync(s->ddesc + r->slot, s->hdesc + r->slot, sizeof(InstanceDesc),
                                            cudaMemcpyHostToDevice, s->s_prep);
            if (e == cudaSuccess)
                e = launch_fix_init(p->fc, p->q.max_iterations, p->stats_cap, p->counts, p->stats, s->s_prep);
            if (e == cudaSuccess) e = launch_fused_init(p->g, fused_args(p, 0, 0), p->cand, s->s_prep);
            if (e == cudaSuccess) e = cudaEventRecord(r->ev, s->s_prep);
            if (e != cudaSuccess) status = GSC_ERR_CUDA;
        }
        if (status != GSC_OK) {
            cudaStreamSynchronize(s->s_prep);
            release(s, r);
            finish(s, r, status);
            continue;
        }
        r->state = kPrep2;
        s->prep2.push_back(r);
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.device_bytes_in_use = s->pool->used();
        s->st.peak_device_bytes = std::max(s->st.peak_device_bytes, s->st.device_bytes_in_use);
    }
    return any;
}

// PREP2 -> RUN once its set-up has finished on the device.
bool advance_prep2(gsc_server* s, bool& list_dirty) {
    bool any = false;
    for (size_t i = 0; i < s->prep2.size();) {
        Req* r = s->prep2[i];
        const cudaError_t q = cudaEventQuery(r->ev);
        if (q == cudaErrorNotReady) {
            ++i;
            continue;
        }
        s->prep2.erase(s->prep2.begin() + i);
        any = true;
        if (q != cudaSuccess) {
            release(s, r);
            finish(s, r, GSC_ERR_CUDA);
            continue;
        }
        r->state = kRun;
        s->running.push_back(r);
        list_dirty = true;
    }
    return any;
}

// A stopped query's results to the caller's buffers, after the step that
// stopped it.
void start_copy(gsc_server* s, Req* r) {
    gsc_problem* p = r->p.get();
    gsc_result* out = r->out;
    const GridInfo& g = p->g;
    cudaStream_t cs = s->s_copy;
    cudaError_t e = cudaSuccess;
    if (out->valid_mask) e = cudaMemcpyAsync(out->valid_mask, p->valid, g.S, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess && out->candidate_mask)
        e = cudaMemcpyAsync(out->candidate_mask, p->cand, g.S, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess && out->reachable_mask) {
        e = launch_unpack_bits(g, (r->fc.iter & 1) ? p->reach1 : p->reach0, p->reach8, cs);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out->reachable_mask, p->reach8, g.S, cudaMemcpyDeviceToHost, cs);
    }
    if (e == cudaSuccess && out->controller)
        e = cudaMemcpyAsync(out->controller, p->controller, g.S * 4, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess && out->reach_step)
        e = cudaMemcpyAsync(out->reach_step, p->reach_step, g.S * 4, cudaMemcpyDeviceToHost, cs);
    const uint32_t rows = std::min<uint32_t>(std::min<uint32_t>(r->fc.iter, out->iter_capacity), kStatsRows - 1);
    if (e == cudaSuccess && rows)
        e = cudaMemcpyAsync(s->hstats + static_cast<size_t>(r->slot) * kStatsRows * kStatsCols, p->stats,
                            sizeof(unsigned long long) * kStatsCols * (rows + 1), cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaEventRecord(r->ev, cs);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(cs);
        release(s, r);
        finish(s, r, GSC_ERR_CUDA);
        return;
    }
    r->state = kCopy;
    s->copying.push_back(r);
}

// COPY -> DONE: summary fields, per-iteration counters, memory and slot back.
bool retire(gsc_server* s) {
    bool any = false;
    for (size_t i = 0; i < s->copying.size();) {
        Req* r = s->copying[i];
        const cudaError_t q = cudaEventQuery(r->ev);
        if (q == cudaErrorNotReady) {
            ++i;
            continue;
        }
        s->copying.erase(s->copying.begin() + i);
        any = true;
        gsc_result* out = r->out;
        const GridInfo& g = r->p->g;
        const FixControl& fc = r->fc;
        for (int d = 0; d < 4; ++d) out->shape[d] = g.n[d];
        out->input_shape[0] = g.ma;
        out->input_shape[1] = g.mw;
        out->states = g.S;
        out->inputs = g.M;
        out->pairs = g.S * g.M;
        out->iterations = fc.iter;
        out->converged = static_cast<int32_t>(fc.converged);
        out->message = static_cast<int32_t>(fc.message ? fc.message : GSC_MSG_MAX_ITERATIONS);
        out->certified_candidates = fc.certified;
        out->reachable_states = fc.reachable;
        out->candidate_count = fc.candidate_count;
        out->valid_count = fc.valid_count;
        const uint32_t rows = std::min<uint32_t>(std::min<uint32_t>(fc.iter, out->iter_capacity), kStatsRows - 1);
        const unsigned long long* hs = s->hstats + static_cast<size_t>(r->slot) * kStatsRows * kStatsCols;
        for (uint32_t k = 0; k < rows; ++k) {
            if (out->iter_new_reachable) out->iter_new_reachable[k] = hs[kStatsCols * (k + 1)];
            if (out->iter_new_certified) out->iter_new_certified[k] = hs[kStatsCols * (k + 1) + 1];
        }
        release(s, r);
        finish(s, r, q == cudaSuccess ? GSC_OK : GSC_ERR_CUDA);
    }
    return any;
}

bool progress(gsc_server* s, bool& list_dirty) {
    bool any = retire(s);
    any |= advance_prep2(s, list_dirty);
    any |= advance_prep1(s);
    any |= admit(s);
    return any;
}

void loop(gsc_server* s) {
    cudaSetDevice(s->ctx->device);
    const int sms = sm_count(s->ctx);
    bool list_dirty = true;
    std::vector<const gsc_problem*> probs, sprobs;
    std::vector<uint32_t> slots, sslots, hl, hls;
    std::vector<BigInstance> big;
    WorkTotals tot{}, tot_small{};
    WorkList wl{}, wl_small{};
    uint32_t wmax = 1;
    size_t smem = 0;
    const uint32_t K = s->opt.iterations_per_step;
    while (true) {
        bool any = progress(s, list_dirty);
        if (s->running.empty()) {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stopping && s->queue.empty() && nothing_in_flight(s)) break;
            if (any) continue;
            if (nothing_in_flight(s) && (s->queue.empty() || s->free_slots.empty()))
                s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            else {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
            continue;
        }
        if (list_dirty) {
            // Queries that fill the GPU alone run the one-problem kernels;
            // the status list covers every running query, in running order.
            probs.clear();
            slots.clear();
            sprobs.clear();
            sslots.clear();
            big.clear();
            uint32_t w = 1;
            smem = 0;
            for (Req* r : s->running) {
                probs.push_back(r->p.get());
                slots.push_back(r->slot);
                if (is_big_instance(r->p->g)) {
                    big.push_back(BigInstance{r->p->g, s->hdesc[r->slot].a});
                    continue;
                }
                sprobs.push_back(r->p.get());
                sslots.push_back(r->slot);
                w = std::max(w, r->p->g.W);
                smem = std::max(smem, instance_smem(r->p.get()));
            }
            wmax = wmax_of(w);
            build_work_list(probs, slots, s->shape.chunk, hl, tot);
            build_work_list(sprobs, sslots, s->shape.chunk, hls, tot_small);
            std::memcpy(s->hlist, hl.data(), hl.size() * 4);
            std::memcpy(s->hlist + hl.size(), hls.data(), hls.size() * 4);
            cudaMemcpyAsync(s->dlist, s->hlist, hl.size() * 4, cudaMemcpyHostToDevice, s->s_main);
            cudaMemcpyAsync(s->dlist_small, s->hlist + hl.size(), hls.size() * 4, cudaMemcpyHostToDevice, s->s_main);
            wl = device_work_list(s->dlist, static_cast<uint32_t>(slots.size()), s->shape.chunk, s->hstatus_dev,
                                  nullptr);
            wl_small = device_work_list(s->dlist_small, static_cast<uint32_t>(sslots.size()), s->shape.chunk, nullptr,
                                        nullptr);
            list_dirty = false;
        }
        const uint32_t n = static_cast<uint32_t>(s->running.size());
        cudaError_t e = cudaSuccess;
        BatchShape shape = s->shape;
        if (batch_sat_smem(shape, smem) > kFusedSmemMax) shape.warp = 0;
        for (uint32_t i = 0; e == cudaSuccess && i < K; ++i)
            e = launch_batch_step(s->ddesc, wl_small, tot_small, wl, big.data(), static_cast<uint32_t>(big.size()),
                                  shape, wmax, smem, sms, 0, 0, s->s_main, nullptr);
        if (e == cudaSuccess) e = cudaEventRecord(s->ev_step, s->s_main);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->st.steps++;
            s->st.max_running = std::max<uint64_t>(s->st.max_running, n);
        }
        // Keep admitting and preparing while the step runs.
        while (e == cudaSuccess) {
            const cudaError_t q = cudaEventQuery(s->ev_step);
            if (q != cudaErrorNotReady) {
                e = q;
                break;
            }
            bool dummy = false;
            if (!retire(s) && !advance_prep1(s) && !admit(s) && !advance_prep2(s, dummy))
                std::this_thread::sleep_for(std::chrono::microseconds(10));
            if (dummy) list_dirty = true;
        }
        if (e != cudaSuccess) {
            // A failed step fails every running query; the loop goes on.
            cudaStreamSynchronize(s->s_main);
            for (Req* r : s->running) {
                release(s, r);
                finish(s, r, GSC_ERR_CUDA);
            }
            s->running.clear();
            list_dirty = true;
            continue;
        }
        // Stopped queries leave the running set; their copies wait for this step.
        bool waited = false;
        std::vector<Req*> keep;
        keep.reserve(n);
        for (uint32_t k = 0; k < n; ++k) {
            Req* r = s->running[k];
            if (!s->hstatus[k].stop) {
                keep.push_back(r);
                continue;
            }
            if (!waited) {
                cudaStreamWaitEvent(s->s_copy, s->ev_step, 0);
                waited = true;
            }
            r->fc = s->hstatus[k];
            start_copy(s, r);
        }
        if (keep.size() != n) {
            // Queries that joined during the step follow the listed ones.
            keep.insert(keep.end(), s->running.begin() + n, s->running.end());
            s->running.swap(keep);
            list_dirty = true;
        }
    }
}

}  // namespace

gsc_server::~gsc_server() {
    // Requests first (their problems release into the pool), then the pool.
    reqs.clear();
    pool.reset();
    if (hdesc) cudaFreeHost(hdesc);
    if (hlist) cudaFreeHost(hlist);
    if (hstatus) cudaFreeHost(hstatus);
    if (hplans) cudaFreeHost(hplans);
    if (hstats) cudaFreeHost(hstats);
    if (dmem) cudaFree(dmem);
    if (ev_step) cudaEventDestroy(ev_step);
    if (s_main) cudaStreamDestroy(s_main);
    if (s_prep) cudaStreamDestroy(s_prep);
    if (s_copy) cudaStreamDestroy(s_copy);
}

extern "C" {

int gsc_server_create(gsc_context* ctx, const gsc_server_options* options, gsc_server** out) {
    if (!ctx || !out) return GSC_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cudaGetLastError();
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    std::unique_ptr<gsc_server> s(new (std::nothrow) gsc_server());
    if (!s) return GSC_ERR_OUT_OF_MEMORY;
    s->ctx = ctx;
    if (options) s->opt = *options;
    gsc_server_options& o = s->opt;
    if (o.max_slots == 0) o.max_slots = 256;
    if (o.iterations_per_step == 0) o.iterations_per_step = 2;
    s->shape.sat_threads = o.sat_threads ? o.sat_threads : 64;
    s->shape.sat_blocks = (o.sat_blocks_per_sm ? o.sat_blocks_per_sm : 16) * static_cast<uint32_t>(sm_count(ctx));
    s->shape.chunk = o.chunk_words ? o.chunk_words : 1024;
    s->shape.warp = o.sat_warp_tasks ? 1u : 0u;
    if (s->shape.sat_threads != 64 && s->shape.sat_threads != 128 && s->shape.sat_threads != 256)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "sat_threads must be 64, 128 or 256");
    if (s->shape.chunk < 256 || s->shape.chunk % 256)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "chunk_words must be a positive multiple of 256");
    if (o.max_slots > 65536) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "max_slots above 65536");
    if (o.memory_budget == 0) {
        size_t fr = 0, total = 0;
        GSC_CU(ctx, cudaMemGetInfo(&fr, &total));
        o.memory_budget = fr / 2;
    }
    s->pool.reset(new DevicePool(ctx, 0, o.memory_budget));
    if (!s->pool->reserve(o.memory_budget))
        return fail(ctx, GSC_ERR_OUT_OF_MEMORY, "server: the memory budget could not be reserved");
    s->ictx.device = ctx->device;
    s->ictx.sm_count = ctx->sm_count;
    GSC_CU(ctx, cudaStreamCreateWithFlags(&s->s_main, cudaStreamNonBlocking));
    GSC_CU(ctx, cudaStreamCreateWithFlags(&s->s_prep, cudaStreamNonBlocking));
    // The copy stream's unpack kernels go ahead of the fixpoint steps' blocks.
    int least = 0, greatest = 0;
    GSC_CU(ctx, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    GSC_CU(ctx, cudaStreamCreateWithPriority(&s->s_copy, cudaStreamNonBlocking, greatest));
    s->ictx.stream = s->s_prep;
    GSC_CU(ctx, cudaEventCreateWithFlags(&s->ev_step, cudaEventDisableTiming));
    const uint32_t n = o.max_slots;
    const size_t list_words = n + 4ull * (n + 1);
    const size_t dbytes = sizeof(InstanceDesc) * n + 2 * 4 * list_words + 256 * 3;
    GSC_CU(ctx, cudaMalloc(&s->dmem, dbytes));
    char* d = static_cast<char*>(s->dmem);
    auto carve = [&](size_t bytes) {
        char* r = d;
        d += (bytes + 255) & ~size_t(255);
        return r;
    };
    s->ddesc = reinterpret_cast<InstanceDesc*>(carve(sizeof(InstanceDesc) * n));
    s->dlist = reinterpret_cast<uint32_t*>(carve(4 * list_words));
    s->dlist_small = reinterpret_cast<uint32_t*>(carve(4 * list_words));
    GSC_CU(ctx, cudaMallocHost(&s->hdesc, sizeof(InstanceDesc) * n));
    GSC_CU(ctx, cudaMallocHost(&s->hlist, 2 * 4 * list_words));
    GSC_CU(ctx, cudaMallocHost(&s->hstatus, sizeof(FixControl) * n));
    GSC_CU(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->hstatus_dev), s->hstatus, 0));
    GSC_CU(ctx, cudaMallocHost(&s->hplans, sizeof(PlanRecord) * n));
    GSC_CU(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->hplans_dev), s->hplans, 0));
    GSC_CU(ctx, cudaMallocHost(&s->hstats, sizeof(unsigned long long) * kStatsCols * kStatsRows * n));
    for (uint32_t i = 0; i < n; ++i) s->free_slots.push_back(n - 1 - i);
    s->st.device_bytes_budget = s->pool->total;
    gsc_server* raw = s.get();
    s->th = std::thread(loop, raw);
    *out = s.release();
    return GSC_OK;
}

int gsc_server_submit(gsc_server* s, const gsc_abstraction* abs, const gsc_query_desc* query, gsc_result* out,
                      uint64_t* ticket) {
    if (!s || !abs || !query || !out || !ticket) return GSC_ERR_INVALID_ARGUMENT;
    if (abs->ctx != s->ctx) return fail(s->ctx, GSC_ERR_INVALID_ARGUMENT, "abstraction belongs to another context");
    std::unique_ptr<Req> r(new (std::nothrow) Req());
    if (!r) return GSC_ERR_OUT_OF_MEMORY;
    r->abs = abs;
    r->q = *query;
    r->out = out;
    r->t_submit = Clock::now();
    if (cudaSetDevice(s->ctx->device) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return GSC_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) {
        cudaEventDestroy(r->ev);
        return GSC_ERR_INVALID_ARGUMENT;
    }
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->queue.push_back(r.get());
    s->reqs.emplace(r->ticket, std::move(r));
    s->st.submitted++;
    s->st.queued++;
    s->st.in_flight++;
    s->cv_work.notify_one();
    return GSC_OK;
}

int gsc_server_wait(gsc_server* s, uint64_t ticket, int32_t timeout_ms, int* status, double* latency_ms) {
    if (!s) return GSC_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return GSC_ERR_INVALID_ARGUMENT;
    Req* r = it->second.get();
    auto done = [r] { return r->state == kDone; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
        return GSC_ERR_TIMEOUT;
    if (status) *status = r->status;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    cudaEventDestroy(r->ev);
    s->reqs.erase(it);
    return GSC_OK;
}

int gsc_server_stats(gsc_server* s, gsc_server_report* out) {
    if (!s || !out) return GSC_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    return GSC_OK;
}

void gsc_server_destroy(gsc_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv_work.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    cudaSetDevice(s->ctx->device);
    for (auto& kv : s->reqs)
        if (kv.second->ev) cudaEventDestroy(kv.second->ev);
    delete s;
}

}  // extern "C"
