// gsc_fixpoint.cu -- the backward-reachability fixpoint on the device.
//
// Reference: the host loop of cuda/kernels.cu:654-767 with
// build_prefix_on_device (:403-484), pair_satisfaction_kernel (:310-336) and
// reduce_inputs_kernel (:338-393); CPU semantics reachability.hpp:53-153.
//
// Semantics kept exactly: Jacobi update (the iteration reads the previous
// reachable set only), controller = lowest satisfied input, reach_step = iter
// for non-candidates, stop rules converged -> stalled -> maximum iterations.
//
// Both methods test a pair by "no valid, not yet reachable cell in the box":
// with D = valid && !reachable and reachable a subset of valid,
// R(box) == V(box) <=> D(box) == 0 (inclusion-exclusion is linear), and
// V(box) > 0 does not change between iterations, so it is folded into the
// pair's validity once.  Equivalently the box count of (reachable || !valid)
// equals the box volume.
//
// Every iteration's kernels first read the control block and return at once
// when a stop rule has fired, so extra queued iterations are no-ops and the
// loop can run as a CUDA graph whose while-condition the control kernel sets.
#include <atomic>

#include "gsc_kernels.cuh"

namespace gsc_b200 {

namespace {

inline unsigned int blocks_for(uint64_t n, int threads) {
    uint64_t b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return static_cast<unsigned int>(b);
}

// Streaming 16-byte load that does not allocate in L1 (the box stream is read
// once per iteration; L1 is kept for the prefix-table gathers).
__device__ __forceinline__ uint4 ld_stream(const uint4* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// ---- 4-D prefix (grid.hpp:253-269 layout, prefix_sum.hpp:15-63 values) -----------------

// Pass along x: one warp per x-row, warp-shuffle inclusive scan with carry.
__global__ void k_prefix_x(GridInfo g, int mode, const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                           int32_t* __restrict__ T, const FixControl* fc) {
    if (fc && fc->stop) return;
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= g.rows) return;
    const uint32_t i1 = static_cast<uint32_t>(warp % g.n[1]);
    const uint64_t q = warp / g.n[1];
    const uint32_t i2 = static_cast<uint32_t>(q % g.n[2]);
    const uint32_t i3 = static_cast<uint32_t>(q / g.n[2]);
    const uint64_t base = static_cast<uint64_t>(i1 + 1) * g.ps[1] + static_cast<uint64_t>(i2 + 1) * g.ps[2] +
                          static_cast<uint64_t>(i3 + 1) * g.ps[3];
    const uint64_t src = warp * g.n[0];
    int32_t carry = 0;
    for (uint32_t x0 = 0; x0 < g.n[0]; x0 += 32) {
        const uint32_t x = x0 + lane;
        int32_t v = 0;
        if (x < g.n[0]) {
            const uint64_t s = src + x;
            v = (mode == 0) ? (a[s] != 0) : (mode == 1) ? (a[s] != 0 && b[s] == 0) : (a[s] == 0);
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int32_t t = __shfl_up_sync(0xFFFFFFFFu, v, off);
            if (lane >= static_cast<uint32_t>(off)) v += t;
        }
        v += carry;
        if (x < g.n[0]) T[base + x + 1] = v;
        carry = __shfl_sync(0xFFFFFFFFu, v, 31);
    }
}

// Pass along dimension dim (1, 2 or 3): one thread per line, lanes along x so
// every step of the line loop is a coalesced row access.
__global__ void k_prefix_axis(GridInfo g, int dim, int32_t* __restrict__ T, const FixControl* fc) {
    if (fc && fc->stop) return;
    const int d1 = (dim == 1) ? 2 : 1;
    const int d2 = (dim == 3) ? 2 : 3;
    const uint64_t lines = static_cast<uint64_t>(g.n[0]) * g.n[d1] * g.n[d2];
    const uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (t >= lines) return;
    const uint32_t x = 1 + static_cast<uint32_t>(t % g.n[0]);
    const uint64_t r = t / g.n[0];
    const uint32_t a1 = 1 + static_cast<uint32_t>(r % g.n[d1]);
    const uint32_t a2 = 1 + static_cast<uint32_t>(r / g.n[d1]);
    const uint64_t idx = x + static_cast<uint64_t>(a1) * g.ps[d1] + static_cast<uint64_t>(a2) * g.ps[d2];
    const uint64_t stride = g.ps[dim];
    int32_t acc = 0;
#pragma unroll 4
    for (uint32_t k = 1; k <= g.n[dim]; ++k) {
        const uint64_t p = idx + k * stride;
        acc += T[p];
        T[p] = acc;
    }
}

// Two-pass build of the same table.  Pass 1 (x and y): one block per
// (theta, v) slice.  Each warp scans rows of the slice's mask along x with
// warp shuffles into shared memory; then one thread per x column scans along
// y and writes the slice's table rows (coalesced along x).
constexpr uint32_t kPrefixXYSmemMax = 96u << 10;
constexpr uint32_t kPrefixZWSmemMax = 32u << 10;

__global__ void __launch_bounds__(256) k_prefix_xy(GridInfo g, int mode, const uint8_t* __restrict__ a,
                                                   const uint8_t* __restrict__ b, int32_t* __restrict__ T,
                                                   const FixControl* fc) {
    if (fc && fc->stop) return;
    extern __shared__ int32_t sxy[];   // [n1][n0]
    const uint32_t n0 = g.n[0], n1 = g.n[1];
    const uint32_t slice = blockIdx.x;   // theta + n2 * v
    const uint32_t z = slice % g.n[2], w = slice / g.n[2];
    const uint32_t cells = n0 * n1;
    const uint64_t src = static_cast<uint64_t>(slice) * cells;
    // The slice's set (one byte per state, contiguous) into shared memory,
    // eight loads in flight per thread.
    constexpr int kU = 8;
    for (uint32_t i0 = threadIdx.x; i0 < cells; i0 += kU * blockDim.x) {
        // Both masks' bytes are loaded before either is tested, so no load
        // waits on another.
        uint32_t av[kU], bv[kU];
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            av[k] = (i < cells) ? a[src + i] : 0u;
            bv[k] = (mode == 1 && i < cells) ? b[src + i] : 0u;
        }
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            const int32_t v = (mode == 0) ? (av[k] != 0) : (mode == 1) ? ((av[k] != 0) & (bv[k] == 0)) : (av[k] == 0);
            if (i < cells) sxy[i] = v;
        }
    }
    __syncthreads();
    // Rows along x: one warp per row, warp-shuffle scans with a carry.
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t y = warp; y < n1; y += nwarps) {
        int32_t carry = 0;
        for (uint32_t x0 = 0; x0 < n0; x0 += 32) {
            const uint32_t x = x0 + lane;
            int32_t v = (x < n0) ? sxy[y * n0 + x] : 0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int32_t t = __shfl_up_sync(0xFFFFFFFFu, v, off);
                if (lane >= static_cast<uint32_t>(off)) v += t;
            }
            v += carry;
            if (x < n0) sxy[y * n0 + x] = v;
            carry = __shfl_sync(0xFFFFFFFFu, v, 31);
        }
    }
    __syncthreads();
    // Columns along y: one thread per x, writing the table rows.
    const uint64_t base = static_cast<uint64_t>(z + 1) * g.ps[2] + static_cast<uint64_t>(w + 1) * g.ps[3] + 1;
    for (uint32_t x = threadIdx.x; x < n0; x += blockDim.x) {
        int32_t acc = 0;
        uint64_t o = base + g.ps[1] + x;
        for (uint32_t y = 0; y < n1; ++y, o += g.ps[1]) {
            acc += sxy[y * n0 + x];
            T[o] = acc;
        }
    }
}

// Pass 2 (theta and v): one block per (tile of 2^lt x cells, y row).  The
// tile's n3 x n2 x 2^lt values are loaded into shared memory (rows of the
// tile are contiguous in the table), scanned along theta by one thread per
// (v, x) line, then along v by one thread per (theta, x) line, which writes
// the table back.
__global__ void __launch_bounds__(256) k_prefix_zw(GridInfo g, uint32_t lt, int32_t* __restrict__ T,
                                                   const FixControl* fc) {
    if (fc && fc->stop) return;
    extern __shared__ int32_t szw[];   // [n3][n2][tw]
    const uint32_t tw = 1u << lt;
    const uint32_t n0 = g.n[0], n2 = g.n[2], n3 = g.n[3];
    const uint32_t tiles = (n0 + tw - 1) >> lt;
    const uint32_t y = blockIdx.x / tiles;
    const uint32_t x0 = (blockIdx.x - y * tiles) << lt;
    const uint32_t nx = min(tw, n0 - x0);
    const uint64_t base = static_cast<uint64_t>(y + 1) * g.ps[1] + x0 + 1;
    const uint32_t cells = (n2 * n3) << lt;
    // The tile into shared memory, eight loads in flight per thread.
    constexpr int kU = 8;
    for (uint32_t i0 = threadIdx.x; i0 < cells; i0 += kU * blockDim.x) {
        int32_t v[kU];
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            const uint32_t tx = i & (tw - 1);
            const uint32_t zw = i >> lt;
            const uint32_t w = zw / n2, z = zw - w * n2;
            v[k] = (i < cells && tx < nx)
                       ? T[base + tx + static_cast<uint64_t>(z + 1) * g.ps[2] + static_cast<uint64_t>(w + 1) * g.ps[3]]
                       : 0;
        }
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const uint32_t i = i0 + k * blockDim.x;
            if (i < cells) szw[i] = v[k];
        }
    }
    __syncthreads();
    for (uint32_t l = threadIdx.x; l < (n3 << lt); l += blockDim.x) {
        const uint32_t tx = l & (tw - 1), w = l >> lt;
        int32_t* q = szw + ((w * n2) << lt) + tx;
        int32_t acc = 0;
        for (uint32_t z = 0; z < n2; ++z) {
            acc += q[z << lt];
            q[z << lt] = acc;
        }
    }
    __syncthreads();
    for (uint32_t l = threadIdx.x; l < (n2 << lt); l += blockDim.x) {
        const uint32_t tx = l & (tw - 1), z = l >> lt;
        if (tx >= nx) continue;
        const int32_t* q = szw + (z << lt) + tx;
        uint64_t o = base + tx + static_cast<uint64_t>(z + 1) * g.ps[2] + g.ps[3];
        int32_t acc = 0;
        for (uint32_t w = 0; w < n3; ++w, o += g.ps[3]) {
            acc += q[(w * n2) << lt];
            T[o] = acc;
        }
    }
}

// ---- stored method ---------------------------------------------------------------------

__device__ __forceinline__ uint32_t q16(const int32_t* __restrict__ P, const GridInfo& g, uint32_t l0, uint32_t l1,
                                        uint32_t l2, uint32_t l3, uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    const uint32_t X[2] = {r0, l0};
    const uint32_t Y[2] = {r1 * g.ps[1], l1 * g.ps[1]};
    const uint32_t Z[2] = {r2 * g.ps[2], l2 * g.ps[2]};
    const uint32_t Wd[2] = {r3 * g.ps[3], l3 * g.ps[3]};
    uint32_t v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m)
        v[m] = static_cast<uint32_t>(__ldg(P + (X[m & 1] + Y[(m >> 1) & 1] + Z[(m >> 2) & 1] + Wd[(m >> 3) & 1])));
    uint32_t t = 0;
#pragma unroll
    for (int m = 0; m < 16; ++m) t = (__popc(m) & 1) ? t - v[m] : t + v[m];
    return t;
}

// D(box) for a packed box (one byte per dimension); a box whose theta range
// crosses the seam is split in two (prefix_sum.hpp:87-105).
__device__ __forceinline__ uint32_t dcount(const int32_t* __restrict__ P, const GridInfo& g, uint32_t lo, uint32_t hi) {
    const uint32_t l0 = lo & 255u, l1 = (lo >> 8) & 255u, l2 = (lo >> 16) & 255u, l3 = lo >> 24;
    const uint32_t r0 = (hi & 255u) + 1, r1 = ((hi >> 8) & 255u) + 1, h2 = (hi >> 16) & 255u, r3 = (hi >> 24) + 1;
    if (l2 <= h2) return q16(P, g, l0, l1, l2, l3, r0, r1, h2 + 1, r3);
    return q16(P, g, l0, l1, l2, l3, r0, r1, g.n[2], r3) + q16(P, g, l0, l1, 0, l3, r0, r1, h2 + 1, r3);
}

// D(box) for a wide box (16 bits per bound).
__device__ __forceinline__ uint32_t dcount16(const int32_t* __restrict__ P, const GridInfo& g, uint4 b) {
    const uint32_t l0 = lo16(b.x), l1 = hi16(b.x), l2 = lo16(b.y), l3 = hi16(b.y);
    const uint32_t r0 = lo16(b.z) + 1, r1 = hi16(b.z) + 1, h2 = lo16(b.w), r3 = hi16(b.w) + 1;
    if (l2 <= h2) return q16(P, g, l0, l1, l2, l3, r0, r1, h2 + 1, r3);
    return q16(P, g, l0, l1, l2, l3, r0, r1, g.n[2], r3) + q16(P, g, l0, l1, 0, l3, r0, r1, h2 + 1, r3);
}

__global__ void k_stored_init(GridInfo g, StoredFixArgs a) {
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint8_t c = a.cand[s];
        a.reach[s] = c ? 1 : 0;
        a.controller[s] = kInvalid32;
        a.reach_step[s] = c ? 0u : kInvalid32;
    }
}

// One thread per two consecutive states: a 16-byte load brings both states'
// boxes for input j (layout boxes[j * S_pad + s]).  Inputs are scanned in
// order and the first satisfied one wins (reachability.hpp:72-107); the
// exists-input reduction of reduce_inputs_kernel (kernels.cu:338-393) is
// fused in, with warp-aggregated counters.
__global__ void __launch_bounds__(256) k_sat_stored(GridInfo g, StoredFixArgs a) {
    const FixControl* fc = a.fc;
    if (fc->stop) return;
    const uint32_t it = fc->iter + 1;
    const uint64_t half = a.S_pad >> 1;
    const uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    unsigned long long nr = 0, nc = 0, nload = 0, ncount = 0;
    if (t < half) {
        bool act[2], isc[2], rch[2], cert[2], found[2] = {false, false};
        uint32_t chosen[2] = {0, 0};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint64_t s = 2 * t + k;
            act[k] = isc[k] = rch[k] = cert[k] = false;
            if (s < g.S) {
                const bool v = a.valid[s] != 0;
                isc[k] = a.cand[s] != 0;
                rch[k] = a.reach[s] != 0;
                cert[k] = a.controller[s] != kInvalid32;
                act[k] = v && !((!isc[k] && rch[k]) || (isc[k] && cert[k]));
            }
        }
        if (act[0] || act[1]) {
            const uint4* bx = reinterpret_cast<const uint4*>(a.boxes) + t;
            uint4 nb = ld_stream(bx);
            for (uint32_t j = 0; j < g.M; ++j) {
                const uint4 b = nb;
                nload += 2;   // one 16-byte load carries two pairs' boxes
                if (j + 1 < g.M) nb = ld_stream(bx + static_cast<uint64_t>(j + 1) * half);
                if (act[0] && !found[0] && b.x != kBoxSentinel) {
                    ++ncount;
                    if (dcount(a.pd, g, b.x, b.y) == 0) {
                        found[0] = true;
                        chosen[0] = j;
                    }
                }
                if (act[1] && !found[1] && b.z != kBoxSentinel) {
                    ++ncount;
                    if (dcount(a.pd, g, b.z, b.w) == 0) {
                        found[1] = true;
                        chosen[1] = j;
                    }
                }
                if ((!act[0] || found[0]) && (!act[1] || found[1])) break;
            }
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (!found[k]) continue;
            const uint64_t s = 2 * t + k;
            if (!rch[k]) {
                a.reach[s] = 1;
                ++nr;
            }
            if (!cert[k]) {
                a.controller[s] = chosen[k];
                if (isc[k])
                    ++nc;
                else
                    a.reach_step[s] = it;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        nr += __shfl_down_sync(0xFFFFFFFFu, nr, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
        nload += __shfl_down_sync(0xFFFFFFFFu, nload, off);
        ncount += __shfl_down_sync(0xFFFFFFFFu, ncount, off);
    }
    if ((threadIdx.x & 31) == 0) {
        unsigned long long* row = a.stats + kStatsCols * it;
        if (nr) atomicAdd(row, nr);
        if (nc) atomicAdd(row + 1, nc);
        if (nload) atomicAdd(row + 2, nload);
        if (ncount) atomicAdd(row + 3, ncount);
    }
}

// The same test on a wide grid (a dimension of more than 255 cells): one
// thread per state, one 16-byte load per input (boxes16[j * S + s]).
__global__ void __launch_bounds__(256) k_sat_stored_wide(GridInfo g, StoredFixArgs a) {
    const FixControl* fc = a.fc;
    if (fc->stop) return;
    const uint32_t it = fc->iter + 1;
    const uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    unsigned long long nr = 0, nc = 0, nload = 0, ncount = 0;
    if (s < g.S) {
        const bool v = a.valid[s] != 0;
        const bool isc = a.cand[s] != 0;
        const bool rch = a.reach[s] != 0;
        const bool cert = a.controller[s] != kInvalid32;
        const bool act = v && !((!isc && rch) || (isc && cert));
        bool found = false;
        uint32_t chosen = 0;
        if (act) {
            const uint4* bx = reinterpret_cast<const uint4*>(a.boxes16) + s;
            uint4 nb = ld_stream(bx);
            for (uint32_t j = 0; j < g.M; ++j) {
                const uint4 b = nb;
                ++nload;
                if (j + 1 < g.M) nb = ld_stream(bx + static_cast<uint64_t>(j + 1) * g.S);
                if (b.x == kBoxSentinel) continue;
                ++ncount;
                if (dcount16(a.pd, g, b) == 0) {
                    found = true;
                    chosen = j;
                    break;
                }
            }
        }
        if (found) {
            if (!rch) {
                a.reach[s] = 1;
                ++nr;
            }
            if (!cert) {
                a.controller[s] = chosen;
                if (isc)
                    ++nc;
                else
                    a.reach_step[s] = it;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        nr += __shfl_down_sync(0xFFFFFFFFu, nr, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
        nload += __shfl_down_sync(0xFFFFFFFFu, nload, off);
        ncount += __shfl_down_sync(0xFFFFFFFFu, ncount, off);
    }
    if ((threadIdx.x & 31) == 0) {
        unsigned long long* row = a.stats + kStatsCols * it;
        if (nr) atomicAdd(row, nr);
        if (nc) atomicAdd(row + 1, nc);
        if (nload) atomicAdd(row + 2, nload);
        if (ncount) atomicAdd(row + 3, ncount);
    }
}

// ---- control (device-side stop rules, reachability.hpp:133-144) -------------------------

__global__ void k_fix_init(FixControl* fc, uint32_t max_iterations, uint32_t stats_cap,
                           const unsigned long long* counts, unsigned long long* stats) {
    const uint32_t n = kStatsCols * stats_cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) stats[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        fc->iter = 0;
        fc->ticket = 0;
        fc->last_new = 0;
        fc->max_iterations = max_iterations;
        fc->stats_cap = stats_cap;
        fc->valid_count = counts[0];
        fc->candidate_count = counts[1];
        fc->certified = 0;
        fc->reachable = counts[1];
        fc->converged = 0;
        fc->stop = (max_iterations == 0) ? 1u : 0u;
        fc->message = (max_iterations == 0) ? 3u : 0u;
    }
}

__global__ void k_control(FixControl* fc, const unsigned long long* stats, cudaGraphConditionalHandle cond,
                          int use_cond, unsigned long long* mirror) {
    if (!fc->stop) {
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
    if (use_cond) cudaGraphSetConditional(cond, fc->stop ? 0u : 1u);
    if (mirror) {
        // iter | stop << 32 for a host loop that polls it.
        *reinterpret_cast<volatile unsigned long long*>(mirror) =
            fc->iter | (static_cast<unsigned long long>(fc->stop ? 1u : 0u) << 32);
        __threadfence_system();
    }
}

__global__ void k_set_condition(const FixControl* fc, cudaGraphConditionalHandle cond) {
    cudaGraphSetConditional(cond, fc->stop ? 0u : 1u);
}

}  // namespace

cudaError_t launch_prefix4(const GridInfo& g, int mode, const uint8_t* a, const uint8_t* b, int32_t* table,
                           const FixControl* ctl, cudaStream_t st, cudaEvent_t* ev) {
    const uint64_t xy_bytes = static_cast<uint64_t>(g.n[0]) * g.n[1] * 4;
    const uint64_t zw_line = static_cast<uint64_t>(g.n[2]) * g.n[3] * 4;
    if (xy_bytes <= kPrefixXYSmemMax && zw_line <= kPrefixZWSmemMax) {
        // Two passes: x and y per (theta, v) slice, then theta and v per
        // (x tile, y) with the widest tile (up to 32 x cells) that fits.
        static std::atomic<bool> configured[64];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64 || !configured[dev].load()) {
            e = cudaFuncSetAttribute(k_prefix_xy, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kPrefixXYSmemMax));
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_prefix_zw, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kPrefixZWSmemMax));
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) configured[dev].store(true);
        }
        uint32_t lt = 5;
        while (lt > 0 && (zw_line << lt) > kPrefixZWSmemMax) --lt;
        k_prefix_xy<<<g.slices, 256, static_cast<size_t>(xy_bytes), st>>>(g, mode, a, b, table, ctl);
        if (ev) cudaEventRecord(ev[0], st);
        const uint32_t tiles = (g.n[0] + (1u << lt) - 1) >> lt;
        k_prefix_zw<<<tiles * g.n[1], 256, static_cast<size_t>(zw_line << lt), st>>>(g, lt, table, ctl);
        if (ev) cudaEventRecord(ev[1], st);
        return cudaGetLastError();
    }
    // Wide slices or theta-v planes: one pass per dimension.
    k_prefix_x<<<blocks_for(g.rows * 32, 256), 256, 0, st>>>(g, mode, a, b, table, ctl);
    if (ev) cudaEventRecord(ev[0], st);
    for (int dim = 1; dim <= 3; ++dim) {
        const int d1 = (dim == 1) ? 2 : 1;
        const int d2 = (dim == 3) ? 2 : 3;
        const uint64_t lines = static_cast<uint64_t>(g.n[0]) * g.n[d1] * g.n[d2];
        k_prefix_axis<<<blocks_for(lines, 256), 256, 0, st>>>(g, dim, table, ctl);
        if (ev) cudaEventRecord(ev[dim], st);
    }
    return cudaGetLastError();
}

__global__ void k_hold(uint64_t ns) {
    uint64_t t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (uint32_t k = 0; k < (1u << 20); ++k) {
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 >= ns) break;
        __nanosleep(128);
    }
}

cudaError_t launch_hold(cudaStream_t st, uint64_t ns) {
    k_hold<<<1, 1, 0, st>>>(ns);
    return cudaGetLastError();
}

cudaError_t launch_stored_init(const GridInfo& g, const StoredFixArgs& a, cudaStream_t st) {
    k_stored_init<<<blocks_for(g.S, 256), 256, 0, st>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_stored_iteration(const GridInfo& g, const StoredFixArgs& a, cudaStream_t st, uint32_t* launches,
                                    cudaEvent_t* ev) {
    if (ev) cudaEventRecord(ev[0], st);
    cudaError_t e = launch_prefix4(g, 1, a.valid, a.reach, a.pd, a.fc, st, ev ? ev + 1 : nullptr);
    if (e != cudaSuccess) return e;
    if (a.wide)
        k_sat_stored_wide<<<blocks_for(g.S, 256), 256, 0, st>>>(g, a);
    else
        k_sat_stored<<<blocks_for(a.S_pad / 2, 256), 256, 0, st>>>(g, a);
    if (ev) cudaEventRecord(ev[5], st);
    k_control<<<1, 1, 0, st>>>(a.fc, a.stats, a.cond, a.use_cond, a.mirror);
    if (ev) cudaEventRecord(ev[6], st);
    if (launches) *launches += prefix4_launches(g) + 2;
    return cudaGetLastError();
}

uint32_t prefix4_launches(const GridInfo& g) {
    const uint64_t xy_bytes = static_cast<uint64_t>(g.n[0]) * g.n[1] * 4;
    const uint64_t zw_line = static_cast<uint64_t>(g.n[2]) * g.n[3] * 4;
    return (xy_bytes <= kPrefixXYSmemMax && zw_line <= kPrefixZWSmemMax) ? 2u : 4u;
}

cudaError_t launch_fix_init(FixControl* fc, uint32_t max_iterations, uint32_t stats_cap,
                            const unsigned long long* counts, unsigned long long* stats, cudaStream_t st) {
    k_fix_init<<<blocks_for(static_cast<uint64_t>(kStatsCols) * stats_cap, 256), 256, 0, st>>>(fc, max_iterations, stats_cap, counts, stats);
    return cudaGetLastError();
}

cudaError_t launch_set_condition(const FixControl* fc, cudaGraphConditionalHandle cond, cudaStream_t st) {
    k_set_condition<<<1, 1, 0, st>>>(fc, cond);
    return cudaGetLastError();
}

}  // namespace gsc_b200
