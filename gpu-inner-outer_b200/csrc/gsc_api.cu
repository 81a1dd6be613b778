// gsc_api.cu -- the C ABI (include/gsc_b200.h) over the sm_100a kernels.
//
// Host-side work mirrors run_case_cuda_u32 (cuda/kernels.cu:492-875), split
// into device-resident stages.  The only host arithmetic on the successor-box
// path is the tabulation of cos/sin along theta trajectories and of the
// theta / v trajectories themselves (model.hpp:26-46), done with the C
// library the reference calls, in its operation order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gsc_internal.hpp"

using namespace gsc_b200;

using namespace gsc_api;

namespace {

constexpr uint32_t kStatsCapMax = 1u << 20;

// Reference wrap_angle (model.hpp:14-24).
double wrap_angle(double x) {
    constexpr double kPi = 3.14159265358979323846;
    constexpr double kTwoPi = 2.0 * kPi;
    while (x < -kPi) x += kTwoPi;
    while (x >= kPi) x -= kTwoPi;
    return x;
}

}  // namespace

namespace gsc_api {

int grid_from_model(const gsc_model_desc* m, GridInfo* g, std::string* err) {
    std::memset(g, 0, sizeof(*g));
    uint64_t total = 1;
    for (int d = 0; d < 4; ++d) {
        if (!(m->state_eta[d] > 0.0)) {
            *err = "state eta must be positive";
            return GSC_ERR_INVALID_ARGUMENT;
        }
        const double width = m->state_ub[d] - m->state_lb[d];
        if (!(width > 0.0)) {
            *err = "state bounds must satisfy ub > lb";
            return GSC_ERR_INVALID_ARGUMENT;
        }
        const double n = std::ceil(width / m->state_eta[d]);
        if (!(n >= 1.0) || n > 65535.0) {
            *err = "state grid dimension out of range (1..65535 cells)";
            return GSC_ERR_UNSUPPORTED;
        }
        g->n[d] = static_cast<uint32_t>(n);
        g->lb[d] = m->state_lb[d];
        g->ub[d] = m->state_ub[d];
        g->eta[d] = m->state_eta[d];
        total *= g->n[d];
    }
    if (total > 0xFFFFFFFFull) {
        *err = "state grid exceeds the selected state index type";
        return GSC_ERR_UNSUPPORTED;
    }
    uint32_t ni[2];
    for (int d = 0; d < 2; ++d) {
        if (!(m->input_eta[d] > 0.0)) {
            *err = "input eta must be positive";
            return GSC_ERR_INVALID_ARGUMENT;
        }
        const double width = m->input_ub[d] - m->input_lb[d];
        if (!(width > 0.0)) {
            *err = "input bounds must satisfy ub > lb";
            return GSC_ERR_INVALID_ARGUMENT;
        }
        const double n = std::ceil(width / m->input_eta[d]);
        if (!(n >= 1.0) || n > 65535.0) {
            *err = "input grid dimension out of range";
            return GSC_ERR_UNSUPPORTED;
        }
        ni[d] = static_cast<uint32_t>(n);
        g->ilb[d] = m->input_lb[d];
        g->ieta[d] = m->input_eta[d];
    }
    if (m->wrap_dim != 2) {
        *err = "only wrap_dim = 2 (theta) is supported";
        return GSC_ERR_UNSUPPORTED;
    }
    if (m->integration_substeps == 0) {
        *err = "integration_substeps must be positive";
        return GSC_ERR_INVALID_ARGUMENT;
    }
    g->ma = ni[0];
    g->mw = ni[1];
    g->M = ni[0] * ni[1];
    g->T = m->sample_time;
    g->K = m->integration_substeps;
    g->dt = m->sample_time / static_cast<double>(m->integration_substeps);
    g->S = total;
    g->ps[0] = 1;
    for (int d = 1; d < 4; ++d) g->ps[d] = g->ps[d - 1] * (g->n[d - 1] + 1);
    g->tsize = static_cast<uint64_t>(g->ps[3]) * (g->n[3] + 1);
    if (g->tsize >= 0x7FFFFFFFull) {
        *err = "padded prefix table exceeds int32 indexing";
        return GSC_ERR_UNSUPPORTED;
    }
    g->W = (g->n[0] + kBits - 1) / kBits;
    g->rows = static_cast<uint64_t>(g->n[1]) * g->n[2] * g->n[3];
    g->slices = g->n[2] * g->n[3];
    g->magic_n1 = fdiv_magic(g->n[1]);
    g->magic_nw = fdiv_magic(g->n[1] * g->W);
    return GSC_OK;
}

int device_alloc(gsc_context* ctx, DevicePool* pool, std::vector<std::pair<void*, uint64_t>>& allocs,
                 uint64_t& bytes, void** p, uint64_t nbytes) {
    *p = nullptr;
    void* q = nullptr;
    if (pool) {
        q = pool->alloc(nbytes);
        if (!q) return fail(ctx, GSC_ERR_OUT_OF_MEMORY, "device memory pool exhausted");
    } else {
        std::lock_guard<std::mutex> lk(ctx->mem_mu);
        if (ctx->budget && ctx->in_use + nbytes > ctx->budget)
            return fail(ctx, GSC_ERR_OUT_OF_MEMORY, "device memory budget exceeded");
        const cudaError_t e = cudaMalloc(&q, nbytes ? nbytes : 1);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, GSC_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        ctx->in_use += nbytes;
    }
    allocs.emplace_back(q, nbytes);
    bytes += nbytes;
    *p = q;
    return GSC_OK;
}

void device_release_all(gsc_context* ctx, DevicePool* pool, std::vector<std::pair<void*, uint64_t>>& allocs,
                        uint64_t& bytes) {
    for (auto& pr : allocs) {
        if (pool) {
            pool->release(pr.first, pr.second);
        } else {
            cudaFree(pr.first);
            if (ctx) ctx->in_use -= pr.second;
        }
    }
    allocs.clear();
    bytes = 0;
}

cudaError_t pinned_get(gsc_context* ctx, size_t bytes, void** p, size_t* got) {
    {
        std::lock_guard<std::mutex> lk(ctx->pin_mu);
        auto it = ctx->pin_free.lower_bound(bytes);
        if (it != ctx->pin_free.end() && it->first <= 2 * bytes + (64u << 10)) {
            *p = it->second;
            *got = it->first;
            ctx->pin_free.erase(it);
            return cudaSuccess;
        }
    }
    *got = bytes;
    return cudaMallocHost(p, bytes);
}

void pinned_put(gsc_context* ctx, void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(ctx->pin_mu);
    ctx->pin_free.emplace(bytes, p);
    size_t held = 0;
    for (const auto& kv : ctx->pin_free) held += kv.first;
    // Past the cap the largest cached blocks go back to the driver.
    while (held > kPinnedCacheMax && !ctx->pin_free.empty()) {
        auto it = std::prev(ctx->pin_free.end());
        held -= it->first;
        cudaFreeHost(it->second);
        ctx->pin_free.erase(it);
    }
}

void pinned_trim(gsc_context* ctx) {
    std::lock_guard<std::mutex> lk(ctx->pin_mu);
    for (auto& kv : ctx->pin_free) cudaFreeHost(kv.second);
    ctx->pin_free.clear();
}

int abstraction_enqueue(gsc_abstraction* a, cudaStream_t st, std::vector<std::pair<void*, uint64_t>>& tmp,
                        cudaEvent_t* h2d_ev) {
    gsc_context* ctx = a->ctx;
    const GridInfo& g = a->g;
    const uint32_t K = g.K;
    // Host tabulation of the theta and v trajectories (model.hpp:34-45).
    std::vector<double> host;   // cos | sin | vseq | thf | vf
    const size_t ncs = static_cast<size_t>(g.n[2]) * g.mw * K, nvs = static_cast<size_t>(g.n[3]) * g.ma * K;
    const size_t nth = static_cast<size_t>(g.n[2]) * g.mw, nvf = static_cast<size_t>(g.n[3]) * g.ma;
    host.resize(2 * ncs + nvs + nth + nvf);
    double* cosT = host.data();
    double* sinT = cosT + ncs;
    double* vseq = sinT + ncs;
    double* thf = vseq + nvs;
    double* vf = thf + nth;
    for (uint32_t i2 = 0; i2 < g.n[2]; ++i2) {
        for (uint32_t jw = 0; jw < g.mw; ++jw) {
            double th = g.lb[2] + (static_cast<double>(i2) + 0.5) * g.eta[2];
            const double omega = g.ilb[1] + (static_cast<double>(jw) + 0.5) * g.ieta[1];
            const size_t base = (static_cast<size_t>(i2) * g.mw + jw) * K;
            for (uint32_t k = 0; k < K; ++k) {
                cosT[base + k] = std::cos(th);
                sinT[base + k] = std::sin(th);
                th = wrap_angle(th + g.dt * omega);
            }
            thf[static_cast<size_t>(i2) * g.mw + jw] = th;
        }
    }
    for (uint32_t i3 = 0; i3 < g.n[3]; ++i3) {
        for (uint32_t ja = 0; ja < g.ma; ++ja) {
            double v = g.lb[3] + (static_cast<double>(i3) + 0.5) * g.eta[3];
            const double acc = g.ilb[0] + (static_cast<double>(ja) + 0.5) * g.ieta[0];
            const size_t base = (static_cast<size_t>(i3) * g.ma + ja) * K;
            for (uint32_t k = 0; k < K; ++k) {
                vseq[base + k] = v;
                v += g.dt * acc;
            }
            vf[static_cast<size_t>(i3) * g.ma + ja] = v;
        }
    }
    const uint64_t planes = static_cast<uint64_t>(g.slices) * g.M;
    void* q = nullptr;
    GSC_TRY(device_alloc(ctx, a->pool, a->allocs, a->bytes, &q, planes * g.n[0] * 8));
    a->xn = static_cast<double*>(q);
    GSC_TRY(device_alloc(ctx, a->pool, a->allocs, a->bytes, &q, planes * g.n[1] * 8));
    a->yn = static_cast<double*>(q);
    GSC_TRY(device_alloc(ctx, a->pool, a->allocs, a->bytes, &q, nth * 8));
    a->thf = static_cast<double*>(q);
    GSC_TRY(device_alloc(ctx, a->pool, a->allocs, a->bytes, &q, nvf * 8));
    a->vf = static_cast<double*>(q);
    uint64_t tmp_bytes = 0;
    GSC_TRY(device_alloc(ctx, a->pool, tmp, tmp_bytes, &q, (2 * ncs + nvs) * 8));
    double* d_tab = static_cast<double*>(q);
    // One upload of the trajectory tables; cudaMemcpyAsync from pageable
    // memory has returned once the source may be reused.
    if (h2d_ev) GSC_CU(ctx, cudaEventRecord(h2d_ev[0], st));
    GSC_CU(ctx, cudaMemcpyAsync(d_tab, cosT, (2 * ncs + nvs) * 8, cudaMemcpyHostToDevice, st));
    GSC_CU(ctx, cudaMemcpyAsync(a->thf, thf, nth * 8, cudaMemcpyHostToDevice, st));
    GSC_CU(ctx, cudaMemcpyAsync(a->vf, vf, nvf * 8, cudaMemcpyHostToDevice, st));
    if (h2d_ev) GSC_CU(ctx, cudaEventRecord(h2d_ev[1], st));
    GSC_CU(ctx, launch_nominal_xy(g, d_tab, d_tab + ncs, d_tab + 2 * ncs, a->xn, a->yn, st));
    return GSC_OK;
}

int sm_count(gsc_context* ctx) { return ctx->sm_count > 0 ? ctx->sm_count : 148; }

// The stored method takes every grid whose bounds fit 16 bits and whose
// padded prefix table is indexed in 32 bits (the reference's own StateIndex
// is 32-bit, grid.hpp:135).
bool stored_fits(const GridInfo& g) {
    return g.n[0] <= 65535 && g.n[1] <= 65535 && g.n[2] <= 65535 && g.n[3] <= 65535 && g.tsize < 0xFFFFFFFFull;
}

// The context's profiling events, created at first use.
cudaError_t profile_events(gsc_context* ctx, cudaEvent_t** out) {
    for (auto& e : ctx->pev)
        if (!e) {
            const cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return err;
        }
    *out = ctx->pev;
    return cudaSuccess;
}

// How long a profiled iteration's launches wait behind launch_hold: more
// than the host takes to queue an iteration's kernels, events and copy.
constexpr uint64_t kProfileHoldNs = 60000;

// The mapped mirror word of host-loop solves.
static cudaError_t loop_resources(gsc_context* ctx) {
    if (ctx->loop_word) return cudaSuccess;
    void* h = nullptr;
    cudaError_t err = cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable);
    if (err != cudaSuccess) return err;
    void* d = nullptr;
    err = cudaHostGetDevicePointer(&d, h, 0);
    if (err != cudaSuccess) {
        cudaFreeHost(h);
        return err;
    }
    ctx->loop_word = static_cast<unsigned long long*>(h);
    ctx->loop_word_dev = static_cast<unsigned long long*>(d);
    return cudaSuccess;
}

// One pause of a host spin-wait.
static inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
    __builtin_ia32_pause();
#endif
}



// Device memory in use on the current GPU (all processes), as the reference
// samples it (kernels.cu:30-42).
uint64_t device_used_bytes() {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return static_cast<uint64_t>(tot - fr);
}

}  // namespace gsc_api

DevicePool::~DevicePool() {
    for (auto& s : slabs) {
        cudaFree(s.base);
        if (ctx) ctx->in_use -= s.bytes;
    }
}

bool DevicePool::reserve(uint64_t bytes) {
    std::lock_guard<std::mutex> lk(mu);
    const uint64_t n = gsc_b200::RangePool::rounded(bytes);
    {
        std::lock_guard<std::mutex> lk2(ctx->mem_mu);
        if (ctx->budget && ctx->in_use + n > ctx->budget) return false;
        void* q = nullptr;
        if (cudaMalloc(&q, n) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        ctx->in_use += n;
        Slab s;
        s.base = static_cast<char*>(q);
        s.bytes = n;
        s.ranges.reset(n);
        slabs.push_back(std::move(s));
    }
    total += n;
    return true;
}

void* DevicePool::alloc(uint64_t bytes) {
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& s : slabs) {
            const uint64_t off = s.ranges.alloc(bytes);
            if (off != gsc_b200::RangePool::kNone) return s.base + off;
        }
        if (slab_bytes == 0) return nullptr;
    }
    const uint64_t need = gsc_b200::RangePool::rounded(bytes);
    if (cap && total + need > cap) return nullptr;
    uint64_t n = std::max(need, slab_bytes);
    if (cap && total + n > cap) n = cap - total;
    // A full-size region when the budget allows it, else one of just this size.
    if (!reserve(n) && (n == need || !reserve(need))) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    const uint64_t off = slabs.back().ranges.alloc(bytes);
    return off == gsc_b200::RangePool::kNone ? nullptr : slabs.back().base + off;
}

void DevicePool::trim() {
    std::lock_guard<std::mutex> lk(mu);
    for (size_t i = 0; i < slabs.size();) {
        if (slabs[i].ranges.used() != 0) {
            ++i;
            continue;
        }
        cudaFree(slabs[i].base);
        if (ctx) ctx->in_use -= slabs[i].bytes;
        total -= slabs[i].bytes;
        slabs.erase(slabs.begin() + i);
    }
}

void DevicePool::release(void* p, uint64_t bytes) {
    std::lock_guard<std::mutex> lk(mu);
    char* c = static_cast<char*>(p);
    for (auto& s : slabs) {
        if (c >= s.base && c < s.base + s.bytes) {
            s.ranges.release(static_cast<uint64_t>(c - s.base), bytes);
            return;
        }
    }
}

uint64_t DevicePool::used() {
    std::lock_guard<std::mutex> lk(mu);
    uint64_t u = 0;
    for (auto& s : slabs) u += s.ranges.used();
    return u;
}

gsc_abstraction::~gsc_abstraction() {
    if (sync_release && ctx) cudaStreamSynchronize(ctx->stream);
    device_release_all(ctx, pool, allocs, bytes);
}

gsc_problem::~gsc_problem() {
    if (sync_release && stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    device_release_all(ctx, pool, allocs, bytes);
}

extern "C" {

int gsc_cuda_backend_compiled(void) { return 1; }

int gsc_abi_version(void) { return GSC_B200_ABI_VERSION; }

const char* gsc_status_string(int status) {
    switch (status) {
        case GSC_OK: return "ok";
        case GSC_ERR_INVALID_ARGUMENT: return "invalid argument";
        case GSC_ERR_CUDA: return "CUDA error";
        case GSC_ERR_OUT_OF_MEMORY: return "out of device memory";
        case GSC_ERR_UNSUPPORTED: return "unsupported";
        case GSC_ERR_NO_DEVICE: return "no CUDA device found";
        case GSC_ERR_CANDIDATE_INVALID: return "candidate set contains invalid states";
        case GSC_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

const char* gsc_message_string(int message) {
    switch (message) {
        case GSC_MSG_CONVERGED: return "all candidate states obtained a controller";
        case GSC_MSG_STALLED: return "iteration stalled before candidate closure";
        case GSC_MSG_MAX_ITERATIONS: return "maximum iterations reached";
        default: return "";
    }
}

int gsc_grid_shape(const gsc_model_desc* model, uint32_t shape[4], uint32_t input_shape[2]) {
    if (!model || !shape || !input_shape) return GSC_ERR_INVALID_ARGUMENT;
    GridInfo g;
    std::string err;
    const int s = grid_from_model(model, &g, &err);
    if (s != GSC_OK) return s;
    for (int d = 0; d < 4; ++d) shape[d] = g.n[d];
    input_shape[0] = g.ma;
    input_shape[1] = g.mw;
    return GSC_OK;
}

int gsc_context_create(int device, void* cuda_stream, gsc_context** out) {
    if (!out) return GSC_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return GSC_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return GSC_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return GSC_ERR_CUDA;
    gsc_context* ctx = new (std::nothrow) gsc_context();
    if (!ctx) return GSC_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    if (cuda_stream) {
        ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return GSC_ERR_CUDA;
        }
        ctx->own_stream = true;
    }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    ctx->pool.reset(new (std::nothrow) DevicePool(ctx, 64ull << 20, 0));
    if (!ctx->pool) {
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return GSC_ERR_OUT_OF_MEMORY;
    }
    if (cudaEventCreate(&ctx->ev[0]) != cudaSuccess || cudaEventCreate(&ctx->ev[1]) != cudaSuccess) {
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return GSC_ERR_CUDA;
    }
    *out = ctx;
    return GSC_OK;
}

void gsc_context_destroy(gsc_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->ev[0]) cudaEventDestroy(ctx->ev[0]);
    if (ctx->ev[1]) cudaEventDestroy(ctx->ev[1]);
    for (auto e : ctx->pev)
        if (e) cudaEventDestroy(e);
    for (auto s : ctx->setup)
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    for (auto e : ctx->setup_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->loop_word) cudaFreeHost(ctx->loop_word);
    ctx->pool.reset();
    pinned_trim(ctx);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int gsc_context_trim(gsc_context* ctx) {
    if (!ctx) return GSC_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return GSC_ERR_CUDA;
    if (ctx->pool) ctx->pool->trim();
    pinned_trim(ctx);
    return GSC_OK;
}

const char* gsc_last_error(const gsc_context* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int gsc_context_set_memory_budget(gsc_context* ctx, uint64_t bytes) {
    if (!ctx) return GSC_ERR_INVALID_ARGUMENT;
    ctx->budget = bytes;
    return GSC_OK;
}

uint64_t gsc_context_memory_in_use(const gsc_context* ctx) { return ctx ? ctx->in_use.load() : 0; }

int gsc_abstraction_create(gsc_context* ctx, const gsc_model_desc* model, gsc_abstraction** out) {
    if (!ctx || !model || !out) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    *out = nullptr;
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    std::unique_ptr<gsc_abstraction> a(new (std::nothrow) gsc_abstraction());
    if (!a) return GSC_ERR_OUT_OF_MEMORY;
    a->ctx = ctx;
    a->model = *model;
    a->pool = ctx->pool.get();
    a->sync_release = true;
    std::string err;
    const int s = grid_from_model(model, &a->g, &err);
    if (s != GSC_OK) return fail(ctx, s, err);
    std::vector<std::pair<void*, uint64_t>> tmp;
    uint64_t tmp_bytes = 0;
    cudaEvent_t* pev = nullptr;
    GSC_CU(ctx, profile_events(ctx, &pev));
    GSC_CU(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    int st = abstraction_enqueue(a.get(), ctx->stream, tmp, pev);
    cudaError_t e = cudaSuccess;
    if (st == GSC_OK) e = cudaEventRecord(ctx->ev[1], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    for (auto& t : tmp) tmp_bytes += t.second;
    device_release_all(ctx, a->pool, tmp, tmp_bytes);
    if (st != GSC_OK) return st;
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    if (e != cudaSuccess)
        return fail(ctx, e == cudaErrorMemoryAllocation ? GSC_ERR_OUT_OF_MEMORY : GSC_ERR_CUDA,
                    std::string("abstraction: ") + cudaGetErrorString(e));
    a->build_ms = ms;
    if (cudaEventElapsedTime(&ms, pev[0], pev[1]) == cudaSuccess) a->h2d_ms = ms;
    cudaGetLastError();
    *out = a.release();
    return GSC_OK;
}

void gsc_abstraction_destroy(gsc_abstraction* a) {
    if (!a) return;
    cudaSetDevice(a->ctx->device);
    delete a;
}

}  // extern "C"

namespace {

}  // namespace

namespace gsc_api {

int problem_stage1(gsc_problem* p, const gsc_query_desc* qd) {
    gsc_context* ctx = p->ctx;
    const GridInfo& g = p->g;
    cudaStream_t st = p->stream;
    const uint32_t method = p->method;
    QueryInfo& q = p->q;
    std::memset(&q, 0, sizeof(q));
    for (int d = 0; d < 4; ++d) {
        q.dhw[d] = qd->disturbance_half_width[d];
        q.cp[d] = qd->constraint_params[d];
        q.map_lb[d] = qd->map_lb[d];
        q.map_ub[d] = qd->map_ub[d];
    }
    if (qd->constraint_kind < 0 || qd->constraint_kind > 3)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "unknown constraint kind");
    if (qd->candidate_kind < 0 || qd->candidate_kind > 1)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "unknown candidate kind");
    if (qd->obstacle_count > 0 && !qd->obstacles) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "obstacles pointer");
    if (qd->safe_mask && qd->safe_mask_rank != 2 && qd->safe_mask_rank != 4)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "safe_mask_rank must be 2 or 4");
    q.ckind = qd->constraint_kind;
    q.n_obstacles = static_cast<int32_t>(qd->obstacle_count);
    q.cand_kind = qd->candidate_kind;
    for (int i = 0; i < 8; ++i) q.cand[i] = qd->candidate[i];
    q.max_iterations = qd->max_iterations;

    // Method pre-check by shape.
    const bool stored_ok = stored_fits(g);
    const bool fused_shape = g.n[0] <= kBits * kMaxWords && g.ma <= 255 && g.n[2] <= 65535 && g.n[3] <= 65535;
    if (method == GSC_METHOD_STORED && !stored_ok)
        return fail(ctx, GSC_ERR_UNSUPPORTED,
                    "stored method needs at most 65535 cells per dimension and a prefix table under 2^32 entries");
    if (method == GSC_METHOD_FUSED && !fused_shape)
        return fail(ctx, GSC_ERR_UNSUPPORTED, "fused method needs at most 256 cells along x");
    if (method > GSC_METHOD_FUSED) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "unknown method");
    p->fused_candidate = method != GSC_METHOD_STORED && fused_shape;

    // Masks.
    GSC_TRY(palloc(p, &p->valid, g.S));
    GSC_TRY(palloc(p, &p->cand, g.S));
    GSC_TRY(palloc(p, &p->counts, 8));
    GSC_TRY(palloc(p, &p->flags, 1));
    GSC_CU(ctx, cudaMemsetAsync(p->counts, 0, 8 * sizeof(unsigned long long), st));
    GSC_CU(ctx, cudaMemsetAsync(p->flags, 0, sizeof(unsigned int), st));
    if (p->time_h2d) GSC_CU(ctx, cudaEventRecord(ctx->pev[0], st));
    if (qd->obstacle_count) {
        GSC_TRY(palloc(p, &p->obstacles, 8ull * qd->obstacle_count));
        GSC_CU(ctx, cudaMemcpyAsync(p->obstacles, qd->obstacles, 64ull * qd->obstacle_count, cudaMemcpyHostToDevice, st));
    }
    if (qd->valid_mask) GSC_CU(ctx, cudaMemcpyAsync(p->valid, qd->valid_mask, g.S, cudaMemcpyHostToDevice, st));
    if (qd->candidate_mask) GSC_CU(ctx, cudaMemcpyAsync(p->cand, qd->candidate_mask, g.S, cudaMemcpyHostToDevice, st));
    if (qd->safe_mask) {
        p->safe_rank = qd->safe_mask_rank;
        const uint64_t n = (p->safe_rank == 4) ? g.S : static_cast<uint64_t>(g.n[0]) * g.n[1];
        GSC_TRY(palloc(p, &p->safe, n));
        GSC_CU(ctx, cudaMemcpyAsync(p->safe, qd->safe_mask, n, cudaMemcpyHostToDevice, st));
    }
    if (p->time_h2d) GSC_CU(ctx, cudaEventRecord(ctx->pev[1], st));
    if (!qd->safe_mask && q.ckind != GSC_CONSTRAINT_NONE) {
        p->safe_rank = 2;
        GSC_TRY(palloc(p, &p->safe, static_cast<uint64_t>(g.n[0]) * g.n[1]));
        GSC_CU(ctx, launch_safe2(g, q, p->safe, st));
    }
    MaskArgs ma{};
    ma.obstacles = p->obstacles;
    ma.valid = p->valid;
    ma.cand = p->cand;
    ma.build_valid = qd->valid_mask ? 0 : 1;
    ma.build_cand = qd->candidate_mask ? 0 : 1;
    ma.safe = qd->safe_mask ? p->safe : nullptr;
    ma.safe_rank = p->safe_rank;
    ma.cmp_safe = p->safe;
    ma.cmp_rank = p->safe_rank;
    ma.counts = p->counts;
    GSC_CU(ctx, launch_masks(g, q, ma, st));

    // Per-axis boxes.
    const uint64_t planes = static_cast<uint64_t>(g.slices) * g.M;
    GSC_TRY(palloc(p, &p->xt, planes * g.n[0]));
    // y tables, class records and dilated rows are read by 16-byte aligned
    // bulk copies up to three words past their last entry: four spare words.
    GSC_TRY(palloc(p, &p->yt, planes * g.n[1] + 4));
    GSC_TRY(palloc(p, &p->zt, static_cast<uint64_t>(g.n[2]) * g.mw));
    GSC_TRY(palloc(p, &p->wt, static_cast<uint64_t>(g.n[3]) * g.ma));
    GSC_CU(ctx, launch_axis_tables(g, q, p->abs->xn, p->abs->yn, p->abs->thf, p->abs->vf, p->xt, p->yt, p->zt, p->wt,
                                   p->flags, st));

    // Fused tables that do not depend on the sets, and the plan.
    GSC_TRY(palloc(p, &p->dplan, 1));
    GSC_CU(ctx, cudaMemsetAsync(p->dplan, 0, sizeof(PlanRecord), st));
    if (p->fused_candidate) {
        GSC_TRY(palloc(p, &p->xcls, planes * class_words(g) + 4));
        GSC_CU(ctx, launch_x_classes(g, p->xt, p->xcls, st));
        GSC_TRY(palloc(p, &p->xrep, planes));
        GSC_CU(ctx, launch_plane_reps(g, p->xt, p->yt, p->wt, p->xrep, &p->dplan->max_reps, st));
        GSC_TRY(palloc(p, &p->kidx, static_cast<uint64_t>(g.n[2]) + 1));
        GSC_TRY(palloc(p, &p->lidx, static_cast<uint64_t>(g.n[3]) + 1));
    }
    GSC_CU(ctx, launch_plan(g, p->zt, p->wt, p->fused_candidate ? p->xrep : nullptr, p->counts, p->flags, p->kidx,
                            p->lidx, p->dplan, st));
    if (!p->hplan) p->hplan = &p->hplan_own;
    if (p->hplan_dev)
        GSC_CU(ctx, launch_store_words(reinterpret_cast<const uint32_t*>(p->dplan),
                                       reinterpret_cast<uint32_t*>(p->hplan_dev), sizeof(PlanRecord) / 4, st));
    else
        GSC_CU(ctx, cudaMemcpyAsync(p->hplan, p->dplan, sizeof(PlanRecord), cudaMemcpyDeviceToHost, st));
    return GSC_OK;
}

int problem_plan(gsc_problem* p) {
    gsc_context* ctx = p->ctx;
    const GridInfo& g = p->g;
    const PlanRecord& pl = *p->hplan;
    if (pl.counts[2] != 0) return fail(ctx, GSC_ERR_CANDIDATE_INVALID, "candidate set contains invalid states");
    p->valid_count = pl.counts[0];
    p->candidate_count = pl.counts[1];
    // need the valid-cell test when some cell's validity is not its safety
    p->need_valid = p->safe ? (pl.counts[4] != 0) : (p->valid_count != g.S);
    const bool stored_ok = stored_fits(g);
    // An empty or over-wide interval, or too many box widths: only the
    // stored count is exact.
    bool fused_ok = p->fused_candidate && pl.fused && pl.flags == 0 && !pl.width_overflow;
    if (fused_ok) {
        p->max_reps = pl.max_reps;
        p->dil = pl.dil;
        // dilated-row offsets are 32-bit in the satisfaction kernel
        if (static_cast<uint64_t>(pl.dil.nk) * pl.dil.nl * g.rows * g.W >= 0xFFFFFFFFull) fused_ok = false;
        if (fused_smem_bytes(g, class_words(g), p->need_valid, p->max_reps, true) > kFusedSmemMax ||
            fused_smem_bytes(g, class_words(g), p->need_valid, p->max_reps, false) > kFusedSmemMax)
            fused_ok = false;
    }
    uint32_t method = p->method;
    if (method == GSC_METHOD_AUTO) method = fused_ok ? GSC_METHOD_FUSED : (stored_ok ? GSC_METHOD_STORED : 0);
    if (method == 0) return fail(ctx, GSC_ERR_UNSUPPORTED, "no method applies to this grid");
    if (method == GSC_METHOD_FUSED && !fused_ok)
        return fail(ctx, GSC_ERR_UNSUPPORTED,
                    "fused method: an interval is empty or wider than 32 cells, or too many box widths");
    p->method = method;
    const uint64_t iter_bound = std::min<uint64_t>(p->q.max_iterations, g.S + 1);
    if (iter_bound + 2 > kStatsCapMax)
        return fail(ctx, GSC_ERR_UNSUPPORTED, "more than 2^20 fixpoint iterations requested");
    p->stats_cap = static_cast<uint32_t>(iter_bound + 2);
    return GSC_OK;
}

int problem_stage2(gsc_problem* p) {
    gsc_context* ctx = p->ctx;
    const GridInfo& g = p->g;
    cudaStream_t st = p->stream;
    GSC_TRY(palloc(p, &p->controller, g.S));
    GSC_TRY(palloc(p, &p->reach_step, g.S));
    GSC_TRY(palloc(p, &p->fc, 1));
    GSC_TRY(palloc(p, &p->stats, static_cast<uint64_t>(kStatsCols) * p->stats_cap));
    GSC_TRY(palloc(p, &p->reach8, g.S));
    // Pool memory is recycled: a read before the first solve sees a zero
    // control record (no iterations), not a previous owner's bytes.
    GSC_CU(ctx, cudaMemsetAsync(p->fc, 0, sizeof(FixControl), st));

    if (p->method == GSC_METHOD_STORED) {
        GSC_TRY(palloc(p, &p->pvalid, g.tsize));
        GSC_CU(ctx, cudaMemsetAsync(p->pvalid, 0, g.tsize * 4, st));
        GSC_CU(ctx, launch_prefix4(g, 0, p->valid, nullptr, p->pvalid, nullptr, st));
        if (p->safe && p->safe_rank == 2) {
            GSC_TRY(palloc(p, &p->unsafe2, static_cast<uint64_t>(g.n[0] + 1) * (g.n[1] + 1)));
            GSC_CU(ctx, launch_prefix2_unsafe(g, p->safe, p->unsafe2, st));
        } else if (p->safe) {
            GSC_TRY(palloc(p, &p->unsafe4, g.tsize));
            GSC_CU(ctx, cudaMemsetAsync(p->unsafe4, 0, g.tsize * 4, st));
            GSC_CU(ctx, launch_prefix4(g, 2, p->safe, nullptr, p->unsafe4, nullptr, st));
        }
        p->S_pad = (g.S + 1) & ~1ull;
        p->wide = g.n[0] > 255 || g.n[1] > 255 || g.n[2] > 255 || g.n[3] > 255;
        if (p->wide)
            GSC_TRY(palloc(p, &p->boxes16, g.S * g.M));
        else
            GSC_TRY(palloc(p, &p->boxes, p->S_pad * g.M));
        StoredBuildArgs sb{};
        sb.xt = p->xt;
        sb.yt = p->yt;
        sb.zt = p->zt;
        sb.wt = p->wt;
        sb.safe = p->safe;
        sb.safe_rank = p->safe_rank;
        sb.unsafe2 = p->unsafe2;
        sb.unsafe4 = p->unsafe4;
        sb.pvalid = p->pvalid;
        sb.boxes = p->boxes;
        sb.S_pad = p->S_pad;
        sb.boxes16 = p->boxes16;
        sb.wide = p->wide ? 1 : 0;
        sb.valid_pairs = p->counts + 3;
        GSC_CU(ctx, launch_stored_build(g, sb, st));
        GSC_TRY(palloc(p, &p->pd, g.tsize));
        GSC_CU(ctx, cudaMemsetAsync(p->pd, 0, g.tsize * 4, st));
        return GSC_OK;
    }
    const uint64_t words = g.rows * g.W;
    GSC_TRY(palloc(p, &p->validb, words));
    GSC_TRY(palloc(p, &p->unsafeb, words));
    GSC_TRY(palloc(p, &p->srcb, words));
    GSC_TRY(palloc(p, &p->candb, words));
    GSC_TRY(palloc(p, &p->dp, words));
    GSC_TRY(palloc(p, &p->reach0, words));
    // One reachable set, updated in place by the finalize: no iteration reads
    // another's reachable words (the satisfaction test reads D' only), so
    // reach1 names the same buffer and every parity choice picks it.
    p->reach1 = p->reach0;
    GSC_TRY(palloc(p, &p->active, words));
    GSC_TRY(palloc(p, &p->hit, words));
    GSC_TRY(palloc(p, &p->best, g.S));
    const uint64_t combos = static_cast<uint64_t>(p->dil.nk) * p->dil.nl;
    GSC_TRY(palloc(p, &p->dzw, combos * words + 4));
    p->rl_words = g.slices * ((g.n[1] + 31) / 32) + 1;
    GSC_TRY(palloc(p, &p->rowlost, 2ull * p->rl_words));
    GSC_TRY(palloc(p, &p->offz, static_cast<uint64_t>(g.n[2]) * g.mw));
    GSC_TRY(palloc(p, &p->offv, static_cast<uint64_t>(g.n[3]) * g.ma));
    GSC_CU(ctx, launch_sat_offsets(g, p->zt, p->wt, p->kidx, p->lidx, p->dil.nl, p->offz, p->offv, st));
    GSC_CU(ctx, launch_pack_bits(g, 0, p->valid, nullptr, p->validb, st));
    GSC_CU(ctx, launch_pack_bits(g, 0, p->cand, nullptr, p->candb, st));
    if (!p->safe) {
        GSC_CU(ctx, cudaMemsetAsync(p->unsafeb, 0, words * sizeof(bword), st));
        GSC_CU(ctx, cudaMemcpyAsync(p->srcb, p->validb, words * sizeof(bword), cudaMemcpyDeviceToDevice, st));
    } else if (p->safe_rank == 2) {
        GSC_CU(ctx, launch_pack_bits(g, 2, nullptr, p->safe, p->unsafeb, st));
        GSC_CU(ctx, launch_pack_bits(g, 3, p->valid, p->safe, p->srcb, st));
    } else {
        GSC_CU(ctx, launch_pack_bits(g, 1, p->safe, nullptr, p->unsafeb, st));
        GSC_CU(ctx, launch_pack_bits(g, 4, p->valid, p->safe, p->srcb, st));
    }
    if (p->need_valid) {
        GSC_TRY(palloc(p, &p->vzw, combos * words + 4));
        GSC_CU(ctx, launch_dilate(g, p->validb, p->vzw, p->dil, nullptr, nullptr, 0, st));
    }
    return GSC_OK;
}

}  // namespace gsc_api

namespace {

StoredFixArgs stored_args(const gsc_problem* p, cudaGraphConditionalHandle cond, int use_cond) {
    StoredFixArgs a{};
    a.boxes = p->boxes;
    a.S_pad = p->S_pad;
    a.boxes16 = p->boxes16;
    a.wide = p->wide ? 1 : 0;
    a.pd = p->pd;
    a.valid = p->valid;
    a.cand = p->cand;
    a.reach = p->reach8;
    a.controller = p->controller;
    a.reach_step = p->reach_step;
    a.fc = p->fc;
    a.stats = p->stats;
    a.cond = cond;
    a.use_cond = use_cond;
    a.mirror = p->mirror;
    return a;
}

}  // namespace

namespace gsc_api {

FusedFixArgs fused_args(const gsc_problem* p, cudaGraphConditionalHandle cond, int use_cond) {
    FusedFixArgs a{};
    a.xt = p->xt;
    a.yt = p->yt;
    a.zt = p->zt;
    a.wt = p->wt;
    a.validb = p->validb;
    a.unsafeb = p->unsafeb;
    a.srcb = p->srcb;
    a.candb = p->candb;
    a.dp = p->dp;
    a.reach0 = p->reach0;
    a.reach1 = p->reach1;
    a.active = p->active;
    a.hit = p->hit;
    a.best = p->best;
    a.controller = p->controller;
    a.reach_step = p->reach_step;
    a.fc = p->fc;
    a.stats = p->stats;
    a.need_valid = p->need_valid;
    a.xcls = p->xcls;
    a.xrep = p->xrep;
    a.cls_words = class_words(p->g);
    a.max_reps = p->max_reps;
    a.sat_threads = fused_sat_threads(p->g, p->max_reps);
    a.dzw = p->dzw;
    a.rowlost = p->rowlost;
    a.shard_begin = p->shard_begin;
    a.shard_slices = p->shard_slices;
    a.rl_words = p->rl_words;
    a.vzw = p->vzw;
    a.kidx = p->kidx;
    a.lidx = p->lidx;
    a.nl = p->dil.nl;
    a.dil = p->dil;
    a.offz = p->offz;
    a.offv = p->offv;
    a.cond = cond;
    a.use_cond = use_cond;
    a.mirror = p->mirror;
    return a;
}

}  // namespace gsc_api

namespace {

cudaError_t enqueue_init(gsc_problem* p) {
    cudaStream_t st = p->ctx->stream;
    cudaError_t e = launch_fix_init(p->fc, p->q.max_iterations, p->stats_cap, p->counts, p->stats, st);
    if (e != cudaSuccess) return e;
    if (p->method == GSC_METHOD_STORED) return launch_stored_init(p->g, stored_args(p, 0, 0), st);
    return launch_fused_init(p->g, fused_args(p, 0, 0), p->cand, st);
}

cudaError_t enqueue_iteration(gsc_problem* p, cudaGraphConditionalHandle cond, int use_cond, uint32_t* launches,
                              cudaEvent_t* ev = nullptr) {
    if (p->method == GSC_METHOD_STORED)
        return launch_stored_iteration(p->g, stored_args(p, cond, use_cond), p->ctx->stream, launches, ev);
    return launch_fused_iteration(p->g, fused_args(p, cond, use_cond), p->ctx->stream, launches, ev);
}

// Outer graph: [init kernels] -> while (condition) { one iteration }.  The
// condition defaults to 1 at each launch; the control kernel at the end of
// the body writes !stop.
int build_graph(gsc_problem* p) {
    gsc_context* ctx = p->ctx;
    cudaStream_t st = ctx->stream;
    cudaGraph_t g = nullptr, ginit = nullptr;
    GSC_CU(ctx, cudaGraphCreate(&g, 0));
    p->graph = g;
    GSC_CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_init(p);
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
    uint32_t launches = 0;
    e = enqueue_iteration(p, handle, 1, &launches);
    cudaGraph_t body_out = nullptr;
    e2 = cudaStreamEndCapture(st, &body_out);
    GSC_CU(ctx, e);
    GSC_CU(ctx, e2);
    GSC_CU(ctx, cudaGraphInstantiate(&p->exec, g, 0));
    return GSC_OK;
}

}  // namespace

extern "C" {

int gsc_problem_create(gsc_context* ctx, const gsc_abstraction* abs, const gsc_query_desc* query, uint32_t method,
                       gsc_problem** out) {
    if (!ctx || !abs || !query || !out) return GSC_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (abs->ctx != ctx) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "abstraction belongs to another context");
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    std::unique_ptr<gsc_problem> p(new (std::nothrow) gsc_problem());
    if (!p) return GSC_ERR_OUT_OF_MEMORY;
    p->ctx = ctx;
    p->abs = abs;
    p->g = abs->g;
    p->stream = ctx->stream;
    p->method = method;
    p->pool = ctx->pool.get();
    p->sync_release = true;
    cudaEvent_t* pev = nullptr;
    GSC_CU(ctx, profile_events(ctx, &pev));
    p->time_h2d = true;
    GSC_CU(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    GSC_TRY(problem_stage1(p.get(), query));
    GSC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    GSC_TRY(problem_plan(p.get()));
    GSC_TRY(problem_stage2(p.get()));
    unsigned long long hc[8];
    GSC_CU(ctx, cudaMemcpyAsync(hc, p->counts, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
    GSC_CU(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    GSC_CU(ctx, cudaEventSynchronize(ctx->ev[1]));
    p->valid_pairs = hc[3];
    float ms = 0.f;
    GSC_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    p->timings.prepare_ms = ms;
    p->timings.abstraction_ms = abs->build_ms;
    if (cudaEventElapsedTime(&ms, pev[0], pev[1]) == cudaSuccess) p->h2d_ms = ms;
    cudaGetLastError();
    p->timings.device_bytes = p->bytes;
    p->timings.method = p->method;
    if (p->method == GSC_METHOD_FUSED) {
        p->timings.max_reps = p->max_reps;
        p->timings.sat_threads = fused_sat_threads(p->g, p->max_reps);
    }
    *out = p.release();
    return GSC_OK;
}

void gsc_problem_destroy(gsc_problem* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    delete p;
}

int gsc_problem_solve(gsc_problem* p, uint32_t flags) {
    if (!p) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    gsc_context* ctx = p->ctx;
    p->shard_begin = p->shard_slices = 0;   // a solve covers the whole grid
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    GSC_CU(ctx, cudaEventRecord(ctx->ev[0], st));
    uint32_t launches = 0;
    double sat_ms = 0.0, scan_ms = 0.0;
    uint32_t sat_launches = 0;
    const uint32_t per_iter = (p->method == GSC_METHOD_STORED) ? prefix4_launches(p->g) + 2 : 3;
    if (flags & GSC_SOLVE_PROFILE) {
        GSC_CU(ctx, enqueue_init(p));
        launches += 2;
        cudaEvent_t* ev = nullptr;
        GSC_CU(ctx, profile_events(ctx, &ev));
        const int npass = p->method == GSC_METHOD_STORED ? static_cast<int>(prefix4_launches(p->g)) : 1;
        for (double& v : p->pass_ms) v = 0.0;
        p->prof_sat_ms = p->prof_reduce_ms = p->prof_memcpy_ms = 0.0;
        p->iter_prof.clear();
        FixControl hfc;
        cudaError_t err = cudaSuccess;
        uint32_t guard = 0;
        while (err == cudaSuccess) {
            // The stop rules fire by iteration stats_cap - 1 at the latest.
            if (++guard > p->stats_cap + 2)
                return fail(ctx, GSC_ERR_TIMEOUT, "fixpoint did not stop within its iteration bound");
            // The hold lets the host queue the iteration and its events
            // before any of them runs.
            err = launch_hold(st, kProfileHoldNs);
            if (err == cudaSuccess) err = enqueue_iteration(p, 0, 0, &launches, ev);
            if (err == cudaSuccess) err = cudaMemcpyAsync(&hfc, p->fc, sizeof(hfc), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess) err = cudaEventRecord(ev[7], st);
            if (err == cudaSuccess) err = cudaStreamSynchronize(st);
            // Events 1 .. npass follow the prefix passes (or the dilation);
            // the satisfaction phase is timed from the last of them.
            float d[kProfileEvents - 1] = {};
            for (int k = 0; err == cudaSuccess && k < kProfileEvents - 1; ++k) {
                if (k >= npass && k < 4) continue;
                err = cudaEventElapsedTime(&d[k], ev[k == 4 ? npass : k], ev[k + 1]);
            }
            if (err != cudaSuccess) break;
            float prefix = 0.f;
            for (int k = 0; k < 4; ++k) {
                p->pass_ms[k] += d[k];
                prefix += d[k];
            }
            scan_ms += prefix;
            sat_ms += d[4];
            p->prof_sat_ms += d[4];
            p->prof_reduce_ms += d[5];
            p->prof_memcpy_ms += d[6];
            p->iter_prof.push_back({prefix + d[4] + d[5] + d[6], prefix, d[4], d[5] + d[6]});
            ++sat_launches;
            if (hfc.stop) break;
        }
        GSC_CU(ctx, err);
    } else if (flags & GSC_SOLVE_GRAPH) {
        if (!p->exec) GSC_TRY(build_graph(p));
        GSC_CU(ctx, cudaGraphLaunch(p->exec, st));
    } else {
        // The host keeps kLoopAhead iterations queued beyond the last one
        // finished, which it reads from the mirror word (written by each
        // iteration's last kernel, no copy in the stream), so the device
        // never waits for the host, and at most kLoopAhead iterations
        // (kernels that return at once on the stop flag) run past the stop.
        // When the stream has drained and the word shows no stop (a stop set
        // by a bounded device wait that gave up), the record in device memory
        // decides.
        constexpr uint32_t kLoopAhead = 2;
        GSC_CU(ctx, loop_resources(ctx));
        volatile unsigned long long* word = ctx->loop_word;
        *word = (p->q.max_iterations == 0) ? (1ull << 32) : 0ull;
        GSC_CU(ctx, enqueue_init(p));
        launches += 2;
        p->mirror = ctx->loop_word_dev;
        uint32_t enq = 0, polls = 0;
        cudaError_t err = cudaSuccess;
        bool timeout = false;
        while (err == cudaSuccess) {
            const unsigned long long m = *word;
            if (m >> 32) break;
            if (enq < static_cast<uint32_t>(m) + kLoopAhead) {
                // The stop rules end the solve by iteration stats_cap - 1.
                if (enq > p->stats_cap + kLoopAhead) {
                    timeout = true;
                    break;
                }
                err = enqueue_iteration(p, 0, 0, &launches);
                ++enq;
                continue;
            }
            if ((++polls & 63) == 0) {
                const cudaError_t q = cudaStreamQuery(st);
                if (q == cudaErrorNotReady) continue;
                if (q != cudaSuccess) {
                    err = q;
                    break;
                }
                FixControl f;
                err = cudaMemcpy(&f, p->fc, sizeof(f), cudaMemcpyDeviceToHost);
                if (err != cudaSuccess || f.stop) break;
                *word = f.iter;
                continue;
            }
            cpu_relax();
        }
        p->mirror = nullptr;
        if (err != cudaSuccess || timeout) cudaStreamSynchronize(st);
        GSC_CU(ctx, err);
        if (timeout) return fail(ctx, GSC_ERR_TIMEOUT, "fixpoint did not stop within its iteration bound");
    }
    GSC_CU(ctx, cudaEventRecord(ctx->ev[1], st));
    GSC_CU(ctx, cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    GSC_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    p->timings.solve_ms = ms;
    // Iteration count and per-iteration counters of this solve.
    FixControl hfc;
    GSC_CU(ctx, cudaMemcpyAsync(&hfc, p->fc, sizeof(hfc), cudaMemcpyDeviceToHost, st));
    GSC_CU(ctx, cudaStreamSynchronize(st));
    std::vector<unsigned long long> hs(static_cast<size_t>(kStatsCols) * (hfc.iter + 1));
    GSC_CU(ctx, cudaMemcpyAsync(hs.data(), p->stats, hs.size() * 8, cudaMemcpyDeviceToHost, st));
    GSC_CU(ctx, cudaStreamSynchronize(st));
    uint64_t tests = 0, aux = 0;
    for (uint32_t i = 1; i <= hfc.iter; ++i) {
        tests += hs[kStatsCols * i + 2];
        aux += hs[kStatsCols * i + 3];
    }
    if (hfc.message == kMsgDeviceTimeout)
        return fail(ctx, GSC_ERR_TIMEOUT, "a bounded device wait for staged rows gave up; the solve stopped");
    p->timings.iterations = hfc.iter;
    p->timings.pair_tests = tests;
    p->timings.aux_count = aux;
    if (flags & GSC_SOLVE_GRAPH && !(flags & GSC_SOLVE_PROFILE))
        launches = 2 + per_iter * std::max<uint32_t>(hfc.iter, 1);   // init child graph + loop bodies
    p->timings.kernel_launches = launches;
    if (flags & GSC_SOLVE_PROFILE) {
        p->timings.sat_kernel_ms = sat_ms;
        p->timings.scan_kernel_ms = scan_ms;
        p->timings.sat_launches = sat_launches;
    }
    return GSC_OK;
}

int gsc_problem_shard_begin(gsc_problem* p, uint32_t slice_begin, uint32_t slice_end) {
    if (!p) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    gsc_context* ctx = p->ctx;
    if (p->method != GSC_METHOD_FUSED) return fail(ctx, GSC_ERR_UNSUPPORTED, "a sharded solve needs the fused method");
    if (slice_begin >= slice_end || slice_end > p->g.slices)
        return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "shard slices out of range");
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    p->shard_begin = 0;
    p->shard_slices = 0;
    GSC_CU(ctx, enqueue_init(p));
    GSC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    p->shard_begin = slice_begin;
    p->shard_slices = slice_end - slice_begin;
    p->shard_iter = 0;
    p->shard_stopped = p->q.max_iterations == 0;
    return GSC_OK;
}

int gsc_problem_shard_step(gsc_problem* p, uint64_t counts[2]) {
    if (!p || !counts) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    gsc_context* ctx = p->ctx;
    if (!p->shard_slices) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "gsc_problem_shard_begin first");
    counts[0] = counts[1] = 0;
    if (p->shard_stopped) return GSC_OK;
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    GSC_CU(ctx, launch_shard_iteration(p->g, fused_args(p, 0, 0), st));
    unsigned long long row[2];
    GSC_CU(ctx, cudaMemcpyAsync(row, p->stats + static_cast<uint64_t>(kStatsCols) * (p->shard_iter + 1), sizeof(row),
                                cudaMemcpyDeviceToHost, st));
    GSC_CU(ctx, cudaStreamSynchronize(st));
    counts[0] = row[0];
    counts[1] = row[1];
    return GSC_OK;
}

int gsc_problem_shard_words(const gsc_problem* p, void** dprime_words, uint64_t* words_per_slice) {
    if (!p || !dprime_words || !words_per_slice) return GSC_ERR_INVALID_ARGUMENT;
    if (p->method != GSC_METHOD_FUSED) return GSC_ERR_UNSUPPORTED;
    *dprime_words = p->dp;
    *words_per_slice = static_cast<uint64_t>(p->g.n[1]) * p->g.W;
    return GSC_OK;
}

int gsc_problem_shard_control(gsc_problem* p, uint64_t new_reachable, uint64_t new_certified, int* stop) {
    if (!p || !stop) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    gsc_context* ctx = p->ctx;
    if (!p->shard_slices) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "gsc_problem_shard_begin first");
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (!p->shard_stopped) GSC_CU(ctx, launch_shard_control(p->fc, p->stats, new_reachable, new_certified, st));
    FixControl fc;
    GSC_CU(ctx, cudaMemcpyAsync(&fc, p->fc, sizeof(fc), cudaMemcpyDeviceToHost, st));
    GSC_CU(ctx, cudaStreamSynchronize(st));
    p->shard_iter = fc.iter;
    p->shard_stopped = fc.stop != 0;
    *stop = p->shard_stopped ? 1 : 0;
    return GSC_OK;
}

int gsc_problem_read(gsc_problem* p, gsc_result* r) {
    if (!p || !r) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    gsc_context* ctx = p->ctx;
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const GridInfo& g = p->g;
    GSC_CU(ctx, cudaEventRecord(ctx->ev[0], st));
    FixControl fc;
    GSC_CU(ctx, cudaMemcpyAsync(&fc, p->fc, sizeof(fc), cudaMemcpyDeviceToHost, st));
    GSC_CU(ctx, cudaStreamSynchronize(st));
    for (int d = 0; d < 4; ++d) r->shape[d] = g.n[d];
    r->input_shape[0] = g.ma;
    r->input_shape[1] = g.mw;
    r->states = g.S;
    r->inputs = g.M;
    r->pairs = g.S * g.M;
    if (fc.message == kMsgDeviceTimeout)
        return fail(ctx, GSC_ERR_TIMEOUT, "the last solve stopped at a bounded device wait that gave up");
    r->iterations = fc.iter;
    r->converged = static_cast<int32_t>(fc.converged);
    r->message = static_cast<int32_t>(fc.message ? fc.message : GSC_MSG_MAX_ITERATIONS);
    r->certified_candidates = fc.certified;
    r->reachable_states = fc.reachable;
    r->candidate_count = fc.candidate_count;
    r->valid_count = fc.valid_count;
    if (r->valid_mask) GSC_CU(ctx, cudaMemcpyAsync(r->valid_mask, p->valid, g.S, cudaMemcpyDeviceToHost, st));
    if (r->candidate_mask) GSC_CU(ctx, cudaMemcpyAsync(r->candidate_mask, p->cand, g.S, cudaMemcpyDeviceToHost, st));
    if (r->reachable_mask) {
        if (p->method == GSC_METHOD_FUSED)
            GSC_CU(ctx, launch_unpack_bits(g, (fc.iter & 1) ? p->reach1 : p->reach0, p->reach8, st));
        GSC_CU(ctx, cudaMemcpyAsync(r->reachable_mask, p->reach8, g.S, cudaMemcpyDeviceToHost, st));
    }
    if (r->controller)
        GSC_CU(ctx, cudaMemcpyAsync(r->controller, p->controller, g.S * 4, cudaMemcpyDeviceToHost, st));
    if (r->reach_step)
        GSC_CU(ctx, cudaMemcpyAsync(r->reach_step, p->reach_step, g.S * 4, cudaMemcpyDeviceToHost, st));
    const uint32_t n = std::min<uint32_t>({fc.iter, r->iter_capacity, p->stats_cap - 1});
    if (n && (r->iter_new_reachable || r->iter_new_certified)) {
        std::vector<unsigned long long> hs(static_cast<size_t>(kStatsCols) * (n + 1));
        GSC_CU(ctx, cudaMemcpyAsync(hs.data(), p->stats, hs.size() * 8, cudaMemcpyDeviceToHost, st));
        GSC_CU(ctx, cudaStreamSynchronize(st));
        for (uint32_t i = 0; i < n; ++i) {
            if (r->iter_new_reachable) r->iter_new_reachable[i] = hs[kStatsCols * (i + 1)];
            if (r->iter_new_certified) r->iter_new_certified[i] = hs[kStatsCols * (i + 1) + 1];
        }
    }
    GSC_CU(ctx, cudaEventRecord(ctx->ev[1], st));
    GSC_CU(ctx, cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    GSC_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    p->timings.readback_ms = ms;
    return GSC_OK;
}

int gsc_problem_export_abstraction(gsc_problem* p, uint32_t* min_flat, uint32_t* max_flat, uint8_t* valid) {
    if (!p || !min_flat || !max_flat || !valid) return GSC_ERR_INVALID_ARGUMENT;
    cudaGetLastError();   // a failure of an unrelated earlier call must not be reported here
    gsc_context* ctx = p->ctx;
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const GridInfo& g = p->g;
    // The export needs the unsafe prefix of the stored build; make it if the
    // fused method skipped it.
    if (p->safe && p->safe_rank == 2 && !p->unsafe2) {
        GSC_TRY(palloc(p, &p->unsafe2, static_cast<uint64_t>(g.n[0] + 1) * (g.n[1] + 1)));
        GSC_CU(ctx, launch_prefix2_unsafe(g, p->safe, p->unsafe2, st));
    } else if (p->safe && p->safe_rank == 4 && !p->unsafe4) {
        GSC_TRY(palloc(p, &p->unsafe4, g.tsize));
        GSC_CU(ctx, cudaMemsetAsync(p->unsafe4, 0, g.tsize * 4, st));
        GSC_CU(ctx, launch_prefix4(g, 2, p->safe, nullptr, p->unsafe4, nullptr, st));
    }
    const uint64_t P = g.S * g.M;
    const uint64_t chunk = std::min<uint64_t>(P, 1ull << 26);
    uint32_t *dmn = nullptr, *dmx = nullptr;
    uint8_t* dv = nullptr;
    cudaError_t e = cudaMalloc(&dmn, chunk * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dmx, chunk * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dv, chunk);
    for (uint64_t b = 0; e == cudaSuccess && b < P; b += chunk) {
        const uint64_t n = std::min<uint64_t>(chunk, P - b);
        ExportArgs ea{};
        ea.xt = p->xt;
        ea.yt = p->yt;
        ea.zt = p->zt;
        ea.wt = p->wt;
        ea.safe = p->safe;
        ea.safe_rank = p->safe_rank;
        ea.unsafe2 = p->unsafe2;
        ea.unsafe4 = p->unsafe4;
        ea.min_flat = dmn;
        ea.max_flat = dmx;
        ea.valid = dv;
        ea.pair_begin = b;
        ea.pair_count = n;
        e = launch_export(g, ea, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(min_flat + b, dmn, n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(max_flat + b, dmx, n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(valid + b, dv, n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFree(dmn);
    cudaFree(dmx);
    cudaFree(dv);
    GSC_CU(ctx, e);
    return GSC_OK;
}

int gsc_problem_timings(const gsc_problem* p, gsc_timings* out) {
    if (!p || !out) return GSC_ERR_INVALID_ARGUMENT;
    *out = p->timings;
    return GSC_OK;
}

namespace {

uint64_t alloc_bytes(const gsc_problem* p, const void* ptr) {
    if (!ptr) return 0;
    for (const auto& a : p->allocs)
        if (a.first == ptr) return a.second;
    return 0;
}

}  // namespace

int gsc_problem_phase_timings(const gsc_problem* p, gsc_phase_timings* out) {
    if (!p || !out) return GSC_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    const gsc_timings& t = p->timings;
    out->abstraction_kernel_ms = t.abstraction_ms + t.prepare_ms;
    out->abstraction_memcpy_h2d_ms = p->abs->h2d_ms + p->h2d_ms;
    out->scatter_mask_ms = 0.0;
    for (int k = 0; k < 4; ++k) out->scan_axis_ms[k] = p->pass_ms[k];
    out->prefix_build_total_ms = p->pass_ms[0] + p->pass_ms[1] + p->pass_ms[2] + p->pass_ms[3];
    out->pair_satisfaction_ms = p->prof_sat_ms;
    out->reduce_inputs_ms = p->prof_reduce_ms;
    out->iteration_memcpy_ms = p->prof_memcpy_ms;
    out->result_memcpy_d2h_ms = t.readback_ms;
    out->total_kernel_ms =
        out->abstraction_kernel_ms + out->prefix_build_total_ms + out->pair_satisfaction_ms + out->reduce_inputs_ms;
    out->total_memcpy_ms = out->abstraction_memcpy_h2d_ms + out->iteration_memcpy_ms + out->result_memcpy_d2h_ms;
    out->total_compute_ms = out->total_kernel_ms + out->total_memcpy_ms;
    // Memory by role, from the problem's own allocations.
    uint64_t boxes = 0;
    for (const void* q : {static_cast<const void*>(p->xt), static_cast<const void*>(p->yt),
                          static_cast<const void*>(p->zt), static_cast<const void*>(p->wt),
                          static_cast<const void*>(p->boxes), static_cast<const void*>(p->boxes16),
                          static_cast<const void*>(p->xcls),
                          static_cast<const void*>(p->xrep), static_cast<const void*>(p->offz),
                          static_cast<const void*>(p->offv), static_cast<const void*>(p->kidx),
                          static_cast<const void*>(p->lidx), static_cast<const void*>(p->unsafe2),
                          static_cast<const void*>(p->unsafe4), static_cast<const void*>(p->safe),
                          static_cast<const void*>(p->obstacles)})
        boxes += alloc_bytes(p, q);
    uint64_t prefix = 0;
    for (const void* q : {static_cast<const void*>(p->pd), static_cast<const void*>(p->pvalid),
                          static_cast<const void*>(p->dzw), static_cast<const void*>(p->vzw),
                          static_cast<const void*>(p->dp), static_cast<const void*>(p->rowlost)})
        prefix += alloc_bytes(p, q);
    out->abstraction_bytes = p->abs->bytes + boxes;
    out->prefix_bytes = prefix;
    out->iteration_bytes = p->bytes - boxes - prefix;
    out->total_allocated_bytes = p->abs->bytes + p->bytes;
    // Sampled here, on demand, rather than on the create / solve path: the
    // query of the driver costs more than a small problem's whole solve.
    out->peak_usage_bytes = std::max(p->peak_used, device_used_bytes());
    out->result_bytes = 11 * p->g.S + 16ull * t.iterations;
    out->profiled_iterations = static_cast<uint32_t>(p->iter_prof.size());
    return GSC_OK;
}

int gsc_problem_iteration_timings(const gsc_problem* p, uint32_t capacity, double* iteration_ms,
                                  double* prefix_build_ms, double* satisfaction_ms, double* reduction_ms) {
    if (!p) return GSC_ERR_INVALID_ARGUMENT;
    const uint32_t n = std::min<uint32_t>(capacity, static_cast<uint32_t>(p->iter_prof.size()));
    for (uint32_t i = 0; i < n; ++i) {
        if (iteration_ms) iteration_ms[i] = p->iter_prof[i][0];
        if (prefix_build_ms) prefix_build_ms[i] = p->iter_prof[i][1];
        if (satisfaction_ms) satisfaction_ms[i] = p->iter_prof[i][2];
        if (reduction_ms) reduction_ms[i] = p->iter_prof[i][3];
    }
    return GSC_OK;
}

int gsc_run_case(int device, const gsc_model_desc* model, const gsc_query_desc* query, uint32_t method,
                 uint32_t flags, gsc_result* out, gsc_timings* timings) {
    if (!model || !query || !out) return GSC_ERR_INVALID_ARGUMENT;
    // One context per device for the one-shot call, kept for the process, so
    // repeated calls reuse its stream and its memory pool; calls on one
    // device are serialised.
    static std::mutex cache_mu;
    static std::map<int, std::pair<gsc_context*, std::unique_ptr<std::mutex>>> cache;
    gsc_context* ctx = nullptr;
    std::mutex* dev_mu = nullptr;
    {
        std::lock_guard<std::mutex> lk(cache_mu);
        auto it = cache.find(device);
        if (it == cache.end()) {
            const int s = gsc_context_create(device, nullptr, &ctx);
            if (s != GSC_OK) return s;
            it = cache.emplace(device, std::make_pair(ctx, std::unique_ptr<std::mutex>(new std::mutex()))).first;
        }
        ctx = it->second.first;
        dev_mu = it->second.second.get();
    }
    std::lock_guard<std::mutex> lk(*dev_mu);
    gsc_abstraction* abs = nullptr;
    gsc_problem* p = nullptr;
    int s = gsc_abstraction_create(ctx, model, &abs);
    if (s == GSC_OK) s = gsc_problem_create(ctx, abs, query, method, &p);
    if (s == GSC_OK) s = gsc_problem_solve(p, flags);
    if (s == GSC_OK) s = gsc_problem_read(p, out);
    if (s == GSC_OK && timings) gsc_problem_timings(p, timings);
    gsc_problem_destroy(p);
    gsc_abstraction_destroy(abs);
    return s;
}

}  // extern "C"
