// gsc_batch_kernels.cu -- the fused fixpoint over many instances at once.
//
// Each kernel is one launch over every listed instance: persistent blocks
// walk a task list (instance k owns tasks off[k] .. off[k+1]-1, found by a
// binary search) and run the same device bodies as the one-problem kernels
// (gsc_fused_body.cuh), so an instance computes the same bits alone and in a
// batch.  Instances that have stopped skip their tasks.  One iteration:
//   k_batch_dilate    (theta, v)-dilated D' of every running instance;
//   k_batch_sat       slice x omega-column tasks of every running instance;
//   k_batch_finalize  word chunks; the last chunk of an instance (ticket)
//                     applies its stop rules;
//   k_batch_status    one block: a copy of every instance's control record,
//                     the number still running, and the CUDA-graph loop
//                     condition.
// Instances big enough to fill the GPU alone run the one-problem kernels in
// the same step (launch_batch_step) and share only init and status.
#include <atomic>

#include "gsc_fused_body.cuh"

namespace gsc_b200 {

using namespace fused;

namespace {

// Largest k in [0, n) with off[k] <= t, given off[0] <= t < off[n].
__device__ __forceinline__ uint32_t find_task(const uint32_t* __restrict__ off, uint32_t n, uint32_t t) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= t)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_batch_init(const InstanceDesc* __restrict__ descs, WorkList wl) {
    const uint32_t total = wl.ini_off[wl.n];
    for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
        const uint32_t k = find_task(wl.ini_off, wl.n, t);
        const InstanceDesc& d = descs[wl.slot[k]];
        const uint64_t b = static_cast<uint64_t>(t - wl.ini_off[k]) * wl.chunk;
        const uint64_t e_end = b + wl.chunk;
        const uint64_t wend = min(e_end, static_cast<uint64_t>(d.words));
        for (uint64_t e = b + threadIdx.x; e < wend; e += blockDim.x) init_word(d.a, e);
        const uint64_t send = min(e_end, d.g.S);
        for (uint64_t s = b + threadIdx.x; s < send; s += blockDim.x) init_state(d.a, d.cand, s);
        const uint64_t tend = min(e_end, static_cast<uint64_t>(kStatsCols) * d.stats_cap);
        for (uint64_t i = b + threadIdx.x; i < tend; i += blockDim.x) d.a.stats[i] = 0;
        if (t == wl.ini_off[k] && threadIdx.x == 0) init_control(d.a.fc, d.max_iterations, d.stats_cap, d.counts);
    }
}

__global__ void __launch_bounds__(256) k_batch_dilate(const InstanceDesc* __restrict__ descs, WorkList wl) {
    const uint32_t total = wl.dil_off[wl.n];
    for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
        const uint32_t k = find_task(wl.dil_off, wl.n, t);
        const InstanceDesc& d = descs[wl.slot[k]];
        if (d.a.fc->stop) continue;
        const uint32_t c = d.a.fc->iter;
        const uint32_t* lost = c > 0 ? d.a.rowlost + (c & 1) * d.a.rl_words : nullptr;
        uint32_t* next = d.a.rowlost + ((c + 1) & 1) * d.a.rl_words;
        const uint32_t b = (t - wl.dil_off[k]) * wl.chunk;
        const uint32_t end = min(b + wl.chunk, d.words);
        // The last task also clears row-bit words beyond the positions.
        const uint32_t span = end == d.words ? max(end, d.a.rl_words) : end;
        for (uint32_t p = b + threadIdx.x; p < span; p += blockDim.x) {
            if (p < d.a.rl_words) next[p] = 0;
            if (p < end) dilate_position(d.g, d.a.dp, d.a.dzw, d.a.dil, p, lost);
        }
    }
}

// The instance of the current task is copied to shared memory when it
// changes; the dynamic shared memory holds the largest instance's staging,
// once per task group.  WARP: every warp of the block walks the task list
// as its own group (tasks blockIdx.x * warps + warp, step gridDim.x *
// warps), else the block is one group.
template <int WMAX, bool WARP>
__global__ void __launch_bounds__(256) k_batch_sat(const InstanceDesc* __restrict__ descs, WorkList wl,
                                                   uint32_t task_words) {
    extern __shared__ __align__(16) bword smem[];
    constexpr uint32_t kGroups = WARP ? 8u : 1u;
    __shared__ __align__(16) InstanceDesc sd[kGroups];
    __shared__ uint32_t s_meta[kGroups][4];
    const uint32_t total = wl.sat_off[wl.n];
    const uint32_t grp = WARP ? (threadIdx.x >> 5) : 0u;
    const uint32_t ngrp = WARP ? (blockDim.x >> 5) : 1u;
    const uint32_t rank = WARP ? (threadIdx.x & 31u) : threadIdx.x;
    const uint32_t gsize = WARP ? 32u : blockDim.x;
    bword* gsm = smem + grp * task_words;
    uint32_t cur = 0xFFFFFFFFu;
    bool stopped = false;
    for (uint32_t t = blockIdx.x * ngrp + grp; t < total; t += gridDim.x * ngrp) {
        const uint32_t k = find_task(wl.sat_off, wl.n, t);
        const uint32_t slot = wl.slot[k];
        if (slot != cur) {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(descs + slot);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sd[grp]);
            for (uint32_t i = rank; i < sizeof(InstanceDesc) / 4; i += gsize) dst[i] = src[i];
            group_sync<WARP>();
            cur = slot;
            // An instance's stop flag changes only in the finalize kernel, so
            // the tasks of a stopped instance are skipped without a look.
            stopped = __ldcg(&sd[grp].a.fc->stop) != 0;
        }
        if (stopped) continue;
        sat_col_task<WMAX, false, 2, WARP>(sd[grp].g, sd[grp].a, t - wl.sat_off[k], gsm, s_meta[grp]);
        group_sync<WARP>();
    }
}

__global__ void __launch_bounds__(256) k_batch_finalize(const InstanceDesc* __restrict__ descs, WorkList wl) {
    __shared__ bool last;
    const uint32_t total = wl.fin_off[wl.n];
    for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
        const uint32_t k = find_task(wl.fin_off, wl.n, t);
        const InstanceDesc& d = descs[wl.slot[k]];
        FixControl* fc = d.a.fc;
        // No chunk of this instance has taken its ticket yet, so its stop
        // flag and iteration cannot change before this task's ticket.
        if (fc->stop) continue;
        const uint32_t it = fc->iter + 1;
        const bword* rprev = (fc->iter & 1) ? d.a.reach1 : d.a.reach0;
        bword* rnext = (fc->iter & 1) ? d.a.reach0 : d.a.reach1;
        const uint64_t b = static_cast<uint64_t>(t - wl.fin_off[k]) * wl.chunk;
        const uint64_t end = min(b + wl.chunk, static_cast<uint64_t>(d.words));
        unsigned long long nr = 0, nc = 0;
        for (uint64_t e = b + threadIdx.x; e < end; e += blockDim.x) finalize_word(d.g, d.a, rprev, rnext, e, it, nr, nc);
        unsigned long long* row = d.a.stats + kStatsCols * it;
        add_counters(row, nr, nc);
        // The counters are atomics; the barrier orders them before the first
        // thread's fence (cumulative) and ticket.
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            last = atomicAdd(&fc->ticket, 1u) == wl.fin_off[k + 1] - wl.fin_off[k] - 1;
        }
        __syncthreads();
        if (last && threadIdx.x == 0) {
            __threadfence();
            fc->ticket = 0;
            control_step(fc, row, it);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_batch_status(const InstanceDesc* __restrict__ descs, WorkList wl,
                                                      cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ uint32_t running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    uint32_t mine = 0;
    for (uint32_t k = threadIdx.x; k < wl.n; k += blockDim.x) {
        const FixControl* fc = descs[wl.slot[k]].a.fc;
        if (wl.status) wl.status[k] = *fc;
        mine += fc->stop ? 0u : 1u;
    }
    if (mine) atomicAdd(&running, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (wl.running) *wl.running = running;
        if (use_cond) cudaGraphSetConditional(cond, running ? 1u : 0u);
    }
}

inline unsigned int grid_of(uint32_t tasks, uint32_t cap) {
    const uint32_t b = tasks < cap ? tasks : cap;
    return b ? b : 1u;
}

template <int WMAX, bool WARP>
cudaError_t launch_sat_t(const InstanceDesc* descs, const WorkList& wl, const WorkTotals& tot, const BatchShape& sh,
                         size_t smem, cudaStream_t st) {
    // Launches may come from several host threads (a server's loop and the
    // caller's); setting the attribute twice is harmless.
    static std::atomic<bool> configured[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !configured[dev].load()) {
        e = cudaFuncSetAttribute(k_batch_sat<WMAX, WARP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kFusedSmemMax));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev].store(true);
    }
    const uint32_t per_block = WARP ? sh.sat_threads / 32 : 1u;
    const uint32_t tasks = (tot.sat + per_block - 1) / per_block;
    const uint32_t blocks = sh.sat_blocks ? grid_of(tasks, sh.sat_blocks) : grid_of(tasks, 0xFFFFFFFFu);
    k_batch_sat<WMAX, WARP><<<blocks, sh.sat_threads, batch_sat_smem(sh, smem), st>>>(
        descs, wl, static_cast<uint32_t>(smem / sizeof(bword)));
    return cudaGetLastError();
}

template <int WMAX>
cudaError_t launch_sat_w(const InstanceDesc* descs, const WorkList& wl, const WorkTotals& tot, const BatchShape& sh,
                         size_t smem, cudaStream_t st) {
    return sh.warp ? launch_sat_t<WMAX, true>(descs, wl, tot, sh, smem, st)
                   : launch_sat_t<WMAX, false>(descs, wl, tot, sh, smem, st);
}

}  // namespace

cudaError_t launch_batch_init(const InstanceDesc* descs, const WorkList& wl, const WorkTotals& tot, int sms,
                              cudaStream_t st) {
    if (tot.ini == 0) return cudaSuccess;
    k_batch_init<<<grid_of(tot.ini, 8u * sms), 256, 0, st>>>(descs, wl);
    return cudaGetLastError();
}

cudaError_t launch_batch_step(const InstanceDesc* descs, const WorkList& small, const WorkTotals& tot_small,
                              const WorkList& all, const BigInstance* big, uint32_t nbig, const BatchShape& sh,
                              uint32_t wmax, size_t smem, int sms, cudaGraphConditionalHandle cond, int use_cond,
                              cudaStream_t st, uint32_t* launches) {
    if (sh.sat_threads < 32 || sh.sat_threads > 256 || sh.sat_threads % 32 || batch_sat_smem(sh, smem) > kFusedSmemMax)
        return cudaErrorInvalidValue;
    uint32_t n = 0;
    cudaError_t e = cudaSuccess;
    // A stopped big instance's kernels return at once (they read its stop flag).
    for (uint32_t i = 0; e == cudaSuccess && i < nbig; ++i) e = launch_fused_iteration(big[i].g, big[i].a, st, &n);
    if (e == cudaSuccess && tot_small.dil) {
        k_batch_dilate<<<grid_of(tot_small.dil, 16u * sms), 256, 0, st>>>(descs, small);
        e = cudaGetLastError();
        ++n;
    }
    if (e == cudaSuccess && tot_small.sat) {
        switch (wmax) {
            case 1: e = launch_sat_w<1>(descs, small, tot_small, sh, smem, st); break;
            case 2: e = launch_sat_w<2>(descs, small, tot_small, sh, smem, st); break;
            case 3:
            case 4: e = launch_sat_w<4>(descs, small, tot_small, sh, smem, st); break;
            default: e = launch_sat_w<8>(descs, small, tot_small, sh, smem, st); break;
        }
        ++n;
    }
    if (e == cudaSuccess && tot_small.fin) {
        k_batch_finalize<<<grid_of(tot_small.fin, 16u * sms), 256, 0, st>>>(descs, small);
        e = cudaGetLastError();
        ++n;
    }
    if (e == cudaSuccess) {
        k_batch_status<<<1, 256, 0, st>>>(descs, all, cond, use_cond);
        e = cudaGetLastError();
        ++n;
    }
    if (launches) *launches += n;
    return e;
}

cudaError_t launch_batch_iteration(const InstanceDesc* descs, const WorkList& wl, const WorkTotals& tot,
                                   const BatchShape& sh, uint32_t wmax, size_t smem, int sms,
                                   cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st,
                                   uint32_t* launches) {
    return launch_batch_step(descs, wl, tot, wl, nullptr, 0, sh, wmax, smem, sms, cond, use_cond, st, launches);
}

}  // namespace gsc_b200
