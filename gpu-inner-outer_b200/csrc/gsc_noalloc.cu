// gsc_noalloc.cu -- a fixpoint entry point that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they need a solve:
// code running inside a pre-planned memory arena (a serving process that has
// already handed every byte of HBM to a pool), plugins loaded into a host
// that owns all allocation, or a hot path that must never hit the driver's
// allocator (cudaMalloc synchronises the device and can fail at any time).
// gsc_fixpoint_noalloc serves them: the caller passes every input and output
// as device memory it already owns, and the working tables the fixpoint
// needs live in one statically sized device array declared in this file.
//
// That array is part of the library's device image: every GPU that loads the
// library holds it until the process exits.  All calls share it, so two calls
// whose work overlaps on the GPU (different streams, different host threads)
// race on it; serialise them.  Each call rewrites every part of the array it
// reads, so what an earlier call left there never leaks into a result.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (a host-side name is not a device address) and caches
// it per device.  Make that first call before any stream capture, since the
// lookup may load the module.  The cached address belongs to the device's
// primary context: after cudaDeviceReset on a device this entry point must not
// be called on that device again in the same process.
//
// Errors: when a launch or copy fails part-way, the call waits for the work it
// already queued on the caller's stream (ignoring that wait's own result)
// before it returns, so nothing it started still touches the shared array or
// the caller's outputs when it returns.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/gsc_b200.h"
#include "gsc_kernels.cuh"

namespace gsc_b200 {
namespace {

// Capacity: the padded prefix table of the grid may have at most
// kNoAllocTableEntries entries ((nx+1)(ny+1)(ntheta+1)(nv+1)); that covers
// the published 70x70x63x13 demo grid and 65x65x38x25.  Iterations are
// bounded by kNoAllocIterations.
constexpr uint64_t kNoAllocTableEntries = 4718592;   // 2^22 + 2^19
constexpr uint32_t kNoAllocIterations = 4096;
constexpr size_t kCtlBytes = 256;
constexpr size_t kStatsBytes = sizeof(unsigned long long) * kStatsCols * (kNoAllocIterations + 2);
constexpr size_t kStatsOffset = kCtlBytes;
constexpr size_t kTableOffset = (kStatsOffset + kStatsBytes + 255) / 256 * 256;
constexpr size_t kTableBytes = kNoAllocTableEntries * sizeof(int32_t);
constexpr size_t kNextOffset = kTableOffset + 2 * kTableBytes;      // next reachable mask (states < entries)
constexpr size_t kScratchBytes = kNextOffset + kNoAllocTableEntries;   // about 40.5 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct NoAllocCtl {
    FixControl fc;
    unsigned long long counts[4];   // [0] valid states, [1] candidate states,
                                    // [2] candidate states that are not valid
};
static_assert(sizeof(NoAllocCtl) <= kCtlBytes, "control block must fit its slot");

std::mutex g_setup_mutex;
void* g_scratch_ptr[64] = {};

int scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GSC_ERR_NO_DEVICE;
    if (dev < 0 || dev >= 64) return GSC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return GSC_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return GSC_OK;
}

__global__ void k_noalloc_init(GridInfo g, const uint8_t* __restrict__ valid, const uint8_t* __restrict__ cand,
                               uint8_t* __restrict__ reach, uint32_t* __restrict__ controller,
                               uint32_t* __restrict__ reach_step, NoAllocCtl* ctl, unsigned long long* stats,
                               uint32_t stats_words) {
    unsigned long long nv = 0, nc = 0, nbad = 0;
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint8_t c = cand[s] ? 1 : 0;
        const bool v = valid[s] != 0;
        reach[s] = c;
        controller[s] = kInvalid32;
        reach_step[s] = c ? 0u : kInvalid32;
        nv += v;
        nc += c;
        nbad += (c && !v);
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < stats_words; i += gridDim.x * blockDim.x) stats[i] = 0;
    for (int off = 16; off > 0; off >>= 1) {
        nv += __shfl_down_sync(0xFFFFFFFFu, nv, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
        nbad += __shfl_down_sync(0xFFFFFFFFu, nbad, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nv) atomicAdd(&ctl->counts[0], nv);
        if (nc) atomicAdd(&ctl->counts[1], nc);
        if (nbad) atomicAdd(&ctl->counts[2], nbad);
    }
}

__global__ void k_noalloc_start(NoAllocCtl* ctl, uint32_t max_iterations, uint32_t stats_cap) {
    FixControl* fc = &ctl->fc;
    fc->iter = 0;
    fc->max_iterations = max_iterations;
    fc->stats_cap = stats_cap;
    fc->valid_count = ctl->counts[0];
    fc->candidate_count = ctl->counts[1];
    fc->certified = 0;
    fc->reachable = ctl->counts[1];
    fc->converged = 0;
    // A candidate set with invalid states is refused before any iteration
    // (abstraction.hpp:268-272); the host turns it into an error status.
    const bool refused = ctl->counts[2] != 0;
    fc->stop = (max_iterations == 0 || refused) ? 1u : 0u;
    fc->message = refused ? 0u : (max_iterations == 0) ? 3u : 0u;
}

__device__ __forceinline__ uint32_t nq16(const int32_t* __restrict__ P, const GridInfo& g, uint32_t l0, uint32_t l1,
                                         uint32_t l2, uint32_t l3, uint32_t r0, uint32_t r1, uint32_t r2,
                                         uint32_t r3) {
    uint32_t t = 0;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const uint32_t x0 = (m & 1) ? l0 : r0;
        const uint32_t x1 = (m & 2) ? l1 : r1;
        const uint32_t x2 = (m & 4) ? l2 : r2;
        const uint32_t x3 = (m & 8) ? l3 : r3;
        const uint32_t v = static_cast<uint32_t>(__ldg(P + x0 + x1 * g.ps[1] + x2 * g.ps[2] + x3 * g.ps[3]));
        t = (__popc(m) & 1) ? t - v : t + v;
    }
    return t;
}

// Box count of a (min_flat, max_flat) pair in the reference's flat layout
// (prefix_sum.hpp:87-105): unflatten both corners, split a theta-wrapped box.
__device__ __forceinline__ uint32_t flat_count(const int32_t* __restrict__ P, const GridInfo& g, uint32_t mn,
                                               uint32_t mx) {
    uint32_t lo[4], hi[4];
    uint32_t v = mn, w = mx;
    for (int d = 0; d < 3; ++d) {
        lo[d] = v % g.n[d];
        v /= g.n[d];
        hi[d] = w % g.n[d];
        w /= g.n[d];
    }
    lo[3] = v;
    hi[3] = w;
    if (lo[2] <= hi[2]) return nq16(P, g, lo[0], lo[1], lo[2], lo[3], hi[0] + 1, hi[1] + 1, hi[2] + 1, hi[3] + 1);
    return nq16(P, g, lo[0], lo[1], lo[2], lo[3], hi[0] + 1, hi[1] + 1, g.n[2], hi[3] + 1) +
           nq16(P, g, lo[0], lo[1], 0, lo[3], hi[0] + 1, hi[1] + 1, hi[2] + 1, hi[3] + 1);
}

// One Jacobi iteration over the caller's abstraction (reachability.hpp:53-109):
// per state, the lowest input whose box has valid_count > 0 and
// reachable_count == valid_count.
__global__ void k_noalloc_iteration(GridInfo g, const uint32_t* __restrict__ min_flat,
                                    const uint32_t* __restrict__ max_flat, const uint8_t* __restrict__ pair_valid,
                                    const uint8_t* __restrict__ valid, const uint8_t* __restrict__ cand,
                                    uint8_t* reach, uint8_t* reach_next, uint32_t* controller, uint32_t* reach_step,
                                    const int32_t* __restrict__ pvalid, const int32_t* __restrict__ preach,
                                    NoAllocCtl* ctl, unsigned long long* stats) {
    const FixControl* fc = &ctl->fc;
    if (fc->stop) return;
    const uint32_t it = fc->iter + 1;
    unsigned long long nr = 0, nc = 0;
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (!valid[s]) continue;
        const bool is_cand = cand[s] != 0;
        const bool reached = reach[s] != 0;
        const bool certified = controller[s] != kInvalid32;
        if ((!is_cand && reached) || (is_cand && certified)) continue;
        const uint64_t base = s * g.M;
        for (uint32_t j = 0; j < g.M; ++j) {
            if (!pair_valid[base + j]) continue;
            const uint32_t vc = flat_count(pvalid, g, min_flat[base + j], max_flat[base + j]);
            if (vc == 0) continue;
            const uint32_t rc = flat_count(preach, g, min_flat[base + j], max_flat[base + j]);
            if (rc != vc) continue;
            if (!reached) {
                reach_next[s] = 1;
                ++nr;
            }
            if (!certified) {
                controller[s] = j;
                if (is_cand)
                    ++nc;
                else
                    reach_step[s] = it;
            }
            break;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        nr += __shfl_down_sync(0xFFFFFFFFu, nr, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nr) atomicAdd(&stats[kStatsCols * it], nr);
        if (nc) atomicAdd(&stats[kStatsCols * it + 1], nc);
    }
}

// reach <- reach_next (the Jacobi swap), then the stop rules
// (reachability.hpp:133-144).
__global__ void k_noalloc_commit(GridInfo g, uint8_t* reach, const uint8_t* __restrict__ reach_next, NoAllocCtl* ctl,
                                 const unsigned long long* stats) {
    if (ctl->fc.stop) return;
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (reach_next[s]) reach[s] = 1;
}

__global__ void k_noalloc_control(NoAllocCtl* ctl, const unsigned long long* stats) {
    FixControl* fc = &ctl->fc;
    if (fc->stop) return;
    const uint32_t it = fc->iter + 1;
    const unsigned long long nr = stats[kStatsCols * it];
    const unsigned long long nc = stats[kStatsCols * it + 1];
    fc->certified += nc;
    fc->reachable += nr;
    fc->iter = it;
    if (fc->certified == fc->candidate_count) {
        fc->converged = 1;
        fc->message = 1;
        fc->stop = 1;
    } else if (nr == 0 && nc == 0) {
        fc->message = 2;
        fc->stop = 1;
    } else if (it >= fc->max_iterations || it + 1 >= fc->stats_cap) {
        fc->message = 3;
        fc->stop = 1;
    }
}

unsigned int nblocks(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    if (b > 65535) b = 65535;
    return static_cast<unsigned int>(b ? b : 1);
}

}  // namespace
}  // namespace gsc_b200

using namespace gsc_b200;

extern "C" int gsc_fixpoint_noalloc(const uint32_t shape[4], uint32_t inputs, int32_t wrap_dim,
                                    const uint32_t* min_flat, const uint32_t* max_flat, const uint8_t* pair_valid,
                                    const uint8_t* valid_mask, const uint8_t* candidate_mask, uint32_t max_iterations,
                                    uint8_t* reachable_mask, uint32_t* controller, uint32_t* reach_step,
                                    gsc_result* summary, void* cuda_stream) {
    if (!shape || !min_flat || !max_flat || !pair_valid || !valid_mask || !candidate_mask || !reachable_mask ||
        !controller || !reach_step || inputs == 0)
        return GSC_ERR_INVALID_ARGUMENT;
    if (wrap_dim != 2) return GSC_ERR_UNSUPPORTED;
    GridInfo g;
    std::memset(&g, 0, sizeof(g));
    uint64_t S = 1, T = 1;
    for (int d = 0; d < 4; ++d) {
        if (shape[d] == 0 || shape[d] > 65535) return GSC_ERR_INVALID_ARGUMENT;
        g.n[d] = shape[d];
        S *= shape[d];
        T *= static_cast<uint64_t>(shape[d]) + 1;
    }
    // Sizes beyond the static scratch are refused before any device work.
    if (T > kNoAllocTableEntries || S > 0xFFFFFFFFull) return GSC_ERR_OUT_OF_MEMORY;
    const uint64_t iter_bound = std::min<uint64_t>(max_iterations, S + 1);
    if (iter_bound + 2 > kNoAllocIterations) return GSC_ERR_OUT_OF_MEMORY;
    g.S = S;
    g.M = inputs;
    g.ps[0] = 1;
    for (int d = 1; d < 4; ++d) g.ps[d] = g.ps[d - 1] * (g.n[d - 1] + 1);
    g.tsize = T;
    g.W = (g.n[0] + 63) / 64;
    g.rows = static_cast<uint64_t>(g.n[1]) * g.n[2] * g.n[3];
    g.slices = g.n[2] * g.n[3];

    unsigned char* base = nullptr;
    const int st_setup = scratch_for_current_device(&base);
    if (st_setup != GSC_OK) return st_setup;
    NoAllocCtl* ctl = reinterpret_cast<NoAllocCtl*>(base);
    unsigned long long* stats = reinterpret_cast<unsigned long long*>(base + kStatsOffset);
    int32_t* pvalid = reinterpret_cast<int32_t*>(base + kTableOffset);
    int32_t* preach = reinterpret_cast<int32_t*>(base + kTableOffset + kTableBytes);
    uint8_t* reachable_next = base + kNextOffset;
    const uint32_t stats_cap = static_cast<uint32_t>(iter_bound + 2);
    const uint32_t stats_words = kStatsCols * stats_cap;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

    // On failure, wait for what this call already queued (its own result is
    // ignored) so that no earlier launch still writes the shared array or the
    // caller's outputs once the call has returned.
#define NA_CU(expr)                                  \
    do {                                             \
        if ((expr) != cudaSuccess) {                 \
            cudaGetLastError();                      \
            cudaStreamSynchronize(st);               \
            cudaGetLastError();                      \
            return GSC_ERR_CUDA;                     \
        }                                            \
    } while (0)

    // Everything read later is rewritten here: the zero planes of both tables,
    // the counters and the control block.
    NA_CU(cudaMemsetAsync(ctl, 0, sizeof(NoAllocCtl), st));
    NA_CU(cudaMemsetAsync(pvalid, 0, T * sizeof(int32_t), st));
    NA_CU(cudaMemsetAsync(preach, 0, T * sizeof(int32_t), st));
    k_noalloc_init<<<nblocks(S), 256, 0, st>>>(g, valid_mask, candidate_mask, reachable_mask, controller, reach_step,
                                                ctl, stats, stats_words);
    NA_CU(cudaGetLastError());
    k_noalloc_start<<<1, 1, 0, st>>>(ctl, max_iterations, stats_cap);
    NA_CU(cudaGetLastError());
    NA_CU(launch_prefix4(g, 0, valid_mask, nullptr, pvalid, nullptr, st));
    NA_CU(cudaMemcpyAsync(reachable_next, reachable_mask, S, cudaMemcpyDeviceToDevice, st));

    NoAllocCtl hc;
    FixControl& h = hc.fc;
    for (;;) {
        for (int k = 0; k < 8; ++k) {
            NA_CU(launch_prefix4(g, 0, reachable_mask, nullptr, preach, &ctl->fc, st));
            k_noalloc_iteration<<<nblocks(S), 256, 0, st>>>(g, min_flat, max_flat, pair_valid, valid_mask,
                                                             candidate_mask, reachable_mask, reachable_next,
                                                             controller, reach_step, pvalid, preach, ctl, stats);
            k_noalloc_commit<<<nblocks(S), 256, 0, st>>>(g, reachable_mask, reachable_next, ctl, stats);
            k_noalloc_control<<<1, 1, 0, st>>>(ctl, stats);
            NA_CU(cudaGetLastError());
        }
        NA_CU(cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, st));
        NA_CU(cudaStreamSynchronize(st));
        if (h.stop) break;
    }
#undef NA_CU
    if (hc.counts[2] != 0) return GSC_ERR_CANDIDATE_INVALID;
    if (summary) {
        for (int d = 0; d < 4; ++d) summary->shape[d] = shape[d];
        summary->states = S;
        summary->inputs = inputs;
        summary->pairs = S * inputs;
        summary->iterations = h.iter;
        summary->converged = static_cast<int32_t>(h.converged);
        summary->message = static_cast<int32_t>(h.message);
        summary->reachable_states = h.reachable;
        summary->certified_candidates = h.certified;
        summary->candidate_count = h.candidate_count;
        summary->valid_count = h.valid_count;
    }
    return GSC_OK;
}
