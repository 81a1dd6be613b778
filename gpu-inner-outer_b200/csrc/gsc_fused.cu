// gsc_fused.cu -- the FUSED fixpoint method: boxes recomputed from per-axis
// tables inside the satisfaction kernel, sets bit-sliced.
//
// Semantics are those of reachability.hpp:53-153 (Jacobi update, lowest
// satisfied input, reach_step = iteration, stop rules in the reference's
// order), as in the stored method.
//
// Data: every set is a bit slice, one 32-bit word per 32 x-cells of a
// (y, theta, v) row.  D' = (valid && !reachable) || unsafe.  A pair is
// satisfied when its box holds no D' cell (so every cell is safe, and every
// valid cell already reachable) and, when validity is more than safety, at
// least one valid cell.
//
// One iteration = three launches:
//   k_dilate         (theta, v)-dilated copies of D' for the box widths in use;
//   k_sat_col        one block per (theta, v) slice x omega column: tests
//                    every active state of the slice against every input of
//                    the column and, per state, records the lowest satisfied
//                    input with an atomicMin into best[] plus a hit bit;
//   k_fused_finalize applies the hits (reachable, active, controller,
//                    reach_step, counters), builds D' for the next iteration,
//                    and its last block applies the stop rules.
#include <atomic>

#include "gsc_fused_body.cuh"

namespace gsc_b200 {

namespace {

inline unsigned int blocks_for(uint64_t n, int threads) {
    uint64_t b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return static_cast<unsigned int>(b);
}

using namespace fused;

__global__ void k_fused_init(GridInfo g, FusedFixArgs a, const uint8_t* __restrict__ cand) {
    const uint64_t words = g.rows * g.W;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < words;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        init_word(a, e);
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        init_state(a, cand, s);
}

// (theta, v)-dilated copies of a bit-sliced set, one thread per word
// position (dilate_position): after the first iteration, with the row-lost
// records, only positions whose widest window holds a row that lost a D'
// cell are recomputed.  The kernel also clears the row bits the next
// finalize writes.
__global__ void k_dilate(GridInfo g, const bword* __restrict__ src, bword* __restrict__ dst, DilateArgs d,
                         const FixControl* fc, uint32_t* rowlost, uint32_t rl_words) {
    pdl_wait();
    if (fc && fc->stop) return;
    const uint32_t c = fc ? fc->iter : 0;
    const uint32_t* lost = (rowlost && c > 0) ? rowlost + (c & 1) * rl_words : nullptr;
    uint32_t* next = rowlost ? rowlost + ((c + 1) & 1) * rl_words : nullptr;
    const uint32_t pos = static_cast<uint32_t>(g.rows * g.W);
    const uint32_t span = next ? max(pos, rl_words) : pos;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < span; p += gridDim.x * blockDim.x) {
        if (next && p < rl_words) next[p] = 0;
        if (p < pos) dilate_position(g, src, dst, d, p, lost);
    }
}

// The set-up plan (one block): which theta widths (wrapped lengths of the
// omega columns' theta boxes) and v widths (of the accelerations' v boxes)
// occur, numbered in increasing order.  out->max_reps (zeroed before, then
// raised by k_plane_reps) becomes at least 1.
__global__ void __launch_bounds__(256) k_plan(GridInfo g, const uint32_t* __restrict__ zt,
                                              const uint32_t* __restrict__ wt, const uint8_t* __restrict__ xrep,
                                              const unsigned long long* __restrict__ counts,
                                              const unsigned int* __restrict__ flags, uint8_t* __restrict__ kidx,
                                              uint8_t* __restrict__ lidx, PlanRecord* __restrict__ out) {
    __shared__ uint32_t kbits[2048], lbits[2048];   // widths 1 .. 65535
    __shared__ DilateArgs s_dil;
    const uint32_t tid = threadIdx.x;
    if (tid < 8) out->counts[tid] = counts[tid];
    if (tid == 0) {
        out->flags = *flags;
        out->fused = xrep ? 1u : 0u;
    }
    if (!xrep) {
        if (tid == 0) {
            out->max_reps = 0;
            out->width_overflow = 0;
            out->dil = DilateArgs{};
        }
        return;
    }
    const uint32_t n2 = g.n[2], n3 = g.n[3];
    for (uint32_t i = tid; i < 2048; i += blockDim.x) kbits[i] = lbits[i] = 0;
    __syncthreads();
    for (uint32_t e = tid; e < n2 * g.mw; e += blockDim.x) {
        const uint32_t ze = zt[e];
        const uint32_t lz = lo16(ze), hz = hi16(ze);
        const uint32_t k = (lz <= hz) ? hz - lz + 1 : n2 - lz + hz + 1;
        atomicOr(&kbits[k >> 5], 1u << (k & 31));
    }
    for (uint32_t e = tid; e < n3 * g.ma; e += blockDim.x) {
        const uint32_t we = wt[e];
        if (we == kReject || hi16(we) < lo16(we)) continue;
        const uint32_t l = hi16(we) - lo16(we) + 1;
        atomicOr(&lbits[l >> 5], 1u << (l & 31));
    }
    __syncthreads();
    if (tid == 0) {
        DilateArgs d{};
        uint32_t over = 0;
        for (uint32_t k = 1; k <= n2; ++k) {
            if (!((kbits[k >> 5] >> (k & 31)) & 1u)) continue;
            if (d.nk == kMaxDilate) {
                over = 1;
                break;
            }
            d.kval[d.nk++] = k;
        }
        for (uint32_t l = 1; l <= n3; ++l) {
            if (!((lbits[l >> 5] >> (l & 31)) & 1u)) continue;
            if (d.nl == kMaxDilate || l > static_cast<uint32_t>(kMaxDilate)) {
                over = 1;
                break;
            }
            d.lval[d.nl++] = l;
        }
        if (d.nk == 0 || d.nl == 0) over = 1;
        s_dil = d;
        out->dil = d;
        out->width_overflow = over;
        out->max_reps = max(out->max_reps, 1u);   // raised by k_plane_reps
    }
    __syncthreads();
    for (uint32_t k = tid; k <= n2; k += blockDim.x) {
        uint32_t slot = 0xFF;
        for (uint32_t i = 0; i < s_dil.nk; ++i)
            if (s_dil.kval[i] == k) slot = i;
        kidx[k] = static_cast<uint8_t>(slot);
    }
    for (uint32_t l = tid; l <= n3; l += blockDim.x) {
        uint32_t slot = 0xFF;
        for (uint32_t i = 0; i < s_dil.nl; ++i)
            if (s_dil.lval[i] == l) slot = i;
        lidx[l] = static_cast<uint8_t>(slot);
    }
}

// The two parts of the word offset in dzw of a representative's dilated D'
// row 0 (sat_col_task, phase B), (kslot * nl + lslot) * rows * W +
// n1 * (lz + n2 * lw) * W in 32-bit arithmetic: per omega column and theta
// cell the kslot and lz terms, per acceleration and v cell the lslot and lw
// terms (0 for a rejected v box, which is never a representative).
__global__ void k_sat_offsets(GridInfo g, const uint32_t* __restrict__ zt, const uint32_t* __restrict__ wt,
                              const uint8_t* __restrict__ kidx, const uint8_t* __restrict__ lidx, uint32_t nl,
                              uint32_t* __restrict__ offz, uint32_t* __restrict__ offv) {
    const uint32_t n1 = g.n[1], n2 = g.n[2], W = g.W;
    const uint32_t pos = static_cast<uint32_t>(g.rows * W);
    const uint32_t nzt = n2 * g.mw, nwt = g.n[3] * g.ma;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nzt + nwt; e += gridDim.x * blockDim.x) {
        if (e < nzt) {
            const uint32_t ze = zt[e];
            const uint32_t lz = lo16(ze), hz = hi16(ze);
            const uint32_t nz = (lz <= hz) ? hz - lz + 1 : n2 - lz + hz + 1;
            offz[e] = kidx[nz] * nl * pos + n1 * lz * W;
        } else {
            const uint32_t we = wt[e - nzt];
            uint32_t o = 0;
            if (we != kReject && hi16(we) >= lo16(we)) {
                const uint32_t lw = lo16(we), nwb = hi16(we) - lw + 1;
                o = lidx[nwb] * pos + n1 * n2 * lw * W;
            }
            offv[e - nzt] = o;
        }
    }
}

// One block per (theta, v) slice x omega column (sat_col_task); a sharded
// solve launches the shard's slices only (task offset shard_begin * mw).
template <int W, bool NV>
__global__ void __launch_bounds__(kFusedWarps * 32) k_sat_col(GridInfo g, FusedFixArgs a) {
    extern __shared__ __align__(16) bword smem[];
    __shared__ uint32_t s_meta[4];
    pdl_wait();
    sat_col_task<W, true, NV ? 1 : 0, false, true>(g, a, blockIdx.x + a.shard_begin * g.mw, smem, s_meta);
}

// Apply the iteration's hits, build next iteration's D', count, and let the
// last block to finish apply the stop rules (reachability.hpp:133-144).  One
// thread per word; the reachable set is updated in place.  A sharded solve
// finalizes the shard's words only and leaves the stop rules to the host,
// which applies them with every rank's counts.
__global__ void __launch_bounds__(256) k_fused_finalize(GridInfo g, FusedFixArgs a) {
    pdl_wait();
    FixControl* fc = a.fc;
    if (fc->stop) {
        // Already stopped (e.g. max_iterations == 0): the graph loop must still end.
        if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
        if (a.mirror && blockIdx.x == 0 && threadIdx.x == 0) write_mirror(a.mirror, fc);
        return;
    }
    const uint32_t it = fc->iter + 1;
    const uint64_t nw = static_cast<uint64_t>(g.n[1]) * g.W;
    const uint64_t first = static_cast<uint64_t>(a.shard_begin) * nw;
    const uint64_t words = a.shard_slices ? a.shard_slices * nw : g.rows * g.W;
    unsigned long long nr = 0, nc = 0;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < words;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        finalize_word(g, a, a.reach0, a.reach0, first + k, it, nr, nc);
    }
    unsigned long long* row = a.stats + kStatsCols * it;
    add_counters(row, nr, nc);
    // Last block to finish: every block's counters are in.  The counters are
    // device-scope atomics; the barrier orders a block's atomics before its
    // first thread's fence (cumulative) and ticket.  Nothing else the last
    // block reads was written by this kernel's other blocks.
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&fc->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x == 0) {
        __threadfence();
        fc->ticket = 0;
        if (a.shard_slices) return;
        control_step(fc, row, it);
        if (a.use_cond) cudaGraphSetConditional(a.cond, fc->stop ? 0u : 1u);
        if (a.mirror) write_mirror(a.mirror, fc);
    }
}

// Stop rules of a sharded iteration with the summed counts of every rank.
__global__ void k_shard_control(FixControl* fc, unsigned long long* stats, unsigned long long nr,
                                unsigned long long nc) {
    if (fc->stop) return;
    const uint32_t it = fc->iter + 1;
    unsigned long long* row = stats + kStatsCols * it;
    row[0] = nr;
    row[1] = nc;
    control_step(fc, row, it);
    fc->last_new = 0xFFFFFFFFu;   // every iteration of a sharded solve tests every pair
}

template <int W, bool NV>
cudaError_t launch_sat_col_t(const GridInfo& g, const FusedFixArgs& a, size_t sm, cudaStream_t st) {
    // Opting in above 48 KB of shared memory is a per-device function attribute.
    // Launches may come from several host threads (a server's loop and the
    // caller's); setting the attribute twice is harmless.
    static std::atomic<bool> configured[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !configured[dev].load()) {
        e = cudaFuncSetAttribute(k_sat_col<W, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kFusedSmemMax));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev].store(true);
    }
    const uint32_t slices = a.shard_slices ? a.shard_slices : g.slices;
    return launch_pdl(k_sat_col<W, NV>, dim3(slices * g.mw), dim3(a.sat_threads), sm, st, g, a);
}

}  // namespace

uint32_t fused_sat_threads(const GridInfo& g, uint32_t max_reps) {
    const uint64_t work = static_cast<uint64_t>(max_reps) * g.n[1] * g.W;
    return work <= 2304 ? 128u : 256u;
}

size_t fused_smem_bytes(const GridInfo& g, uint32_t cls_words, int need_valid, uint32_t max_reps, bool bulk) {
    const FusedSmemLayout L =
        fused_smem_layout(g.n[1] * g.W, need_valid ? 2u : 1u, max_reps, cls_words, g.n[1], g.ma, bulk);
    return sizeof(bword) * static_cast<size_t>(L.total);
}

cudaError_t launch_plan(const GridInfo& g, const uint32_t* zt, const uint32_t* wt, const uint8_t* xrep,
                        const unsigned long long* counts, const unsigned int* flags, uint8_t* kidx, uint8_t* lidx,
                        PlanRecord* out, cudaStream_t st) {
    if (xrep && (g.n[2] > 65535 || g.n[3] > 65535)) return cudaErrorInvalidValue;
    k_plan<<<1, 256, 0, st>>>(g, zt, wt, xrep, counts, flags, kidx, lidx, out);
    return cudaGetLastError();
}

cudaError_t launch_dilate(const GridInfo& g, const bword* src, bword* dst, const DilateArgs& d, const FixControl* fc,
                          uint32_t* rowlost, uint32_t rl_words, cudaStream_t st) {
    const uint64_t pos = g.rows * g.W;
    uint64_t b = (pos + 255) / 256;
    if (b > 8192) b = 8192;
    return launch_pdl(k_dilate, dim3(static_cast<unsigned int>(b ? b : 1)), dim3(256), 0, st, g, src, dst, d, fc,
                      rowlost, rl_words);
}

cudaError_t launch_sat_offsets(const GridInfo& g, const uint32_t* zt, const uint32_t* wt, const uint8_t* kidx,
                               const uint8_t* lidx, uint32_t nl, uint32_t* offz, uint32_t* offv, cudaStream_t st) {
    const uint64_t n = static_cast<uint64_t>(g.n[2]) * g.mw + static_cast<uint64_t>(g.n[3]) * g.ma;
    k_sat_offsets<<<blocks_for(n, 256), 256, 0, st>>>(g, zt, wt, kidx, lidx, nl, offz, offv);
    return cudaGetLastError();
}

cudaError_t launch_fused_init(const GridInfo& g, const FusedFixArgs& a, const uint8_t* cand, cudaStream_t st) {
    k_fused_init<<<blocks_for(g.S, 256), 256, 0, st>>>(g, a, cand);
    return cudaGetLastError();
}

cudaError_t launch_shard_iteration(const GridInfo& g, const FusedFixArgs& a, cudaStream_t st) {
    return launch_fused_iteration(g, a, st, nullptr, nullptr);
}

cudaError_t launch_shard_control(FixControl* fc, unsigned long long* stats, unsigned long long new_reachable,
                                 unsigned long long new_certified, cudaStream_t st) {
    k_shard_control<<<1, 1, 0, st>>>(fc, stats, new_reachable, new_certified);
    return cudaGetLastError();
}

cudaError_t launch_fused_iteration(const GridInfo& g, const FusedFixArgs& a, cudaStream_t st, uint32_t* launches,
                                   cudaEvent_t* ev) {
    if (ev) cudaEventRecord(ev[0], st);
    // A sharded solve dilates the whole grid every iteration: the other
    // ranks' D' slabs arrive without row-lost records.
    cudaError_t derr = launch_dilate(g, a.dp, a.dzw, a.dil, a.fc, a.shard_slices ? nullptr : a.rowlost, a.rl_words, st);
    if (derr != cudaSuccess) return derr;
    if (ev) cudaEventRecord(ev[1], st);
    const size_t sm = fused_smem_bytes(g, a.cls_words, a.need_valid, a.max_reps, true);
    cudaError_t err;
#define GSC_SAT_CASE(Wn)                                                                         \
    case Wn:                                                                                     \
        err = a.need_valid ? launch_sat_col_t<Wn, true>(g, a, sm, st) : launch_sat_col_t<Wn, false>(g, a, sm, st); \
        break;
    switch (g.W) {
        GSC_SAT_CASE(1)
        GSC_SAT_CASE(2)
        GSC_SAT_CASE(3)
        GSC_SAT_CASE(4)
        GSC_SAT_CASE(5)
        GSC_SAT_CASE(6)
        GSC_SAT_CASE(7)
        default:
            err = a.need_valid ? launch_sat_col_t<8, true>(g, a, sm, st) : launch_sat_col_t<8, false>(g, a, sm, st);
            break;
    }
#undef GSC_SAT_CASE
    if (err != cudaSuccess) return err;
    if (ev) cudaEventRecord(ev[5], st);
    const uint64_t words = a.shard_slices ? static_cast<uint64_t>(a.shard_slices) * g.n[1] * g.W : g.rows * g.W;
    uint64_t fb = (words + 255) / 256;
    if (fb > 4096) fb = 4096;
    if (launches) *launches += 3;
    err = launch_pdl(k_fused_finalize, dim3(static_cast<unsigned int>(fb ? fb : 1)), dim3(256), 0, st, g, a);
    if (ev) cudaEventRecord(ev[6], st);
    return err;
}

}  // namespace gsc_b200
