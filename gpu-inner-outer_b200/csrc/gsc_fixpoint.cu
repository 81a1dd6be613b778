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

// ---- control (device-side stop rules, reachability.hpp:133-144) -------------------------

__global__ void k_fix_init(FixControl* fc, uint32_t max_iterations, uint32_t stats_cap,
                           const unsigned long long* counts, unsigned long long* stats) {
    const uint32_t n = kStatsCols * stats_cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) stats[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        fc->iter = 0;
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
                          int use_cond) {
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
}

__global__ void k_set_condition(const FixControl* fc, cudaGraphConditionalHandle cond) {
    cudaGraphSetConditional(cond, fc->stop ? 0u : 1u);
}

// ---- fused method (bit-sliced sets, boxes from per-axis tables) -------------------------

__global__ void k_fused_init(GridInfo g, FusedFixArgs a, const uint8_t* __restrict__ cand) {
    const uint64_t words = g.rows * g.W;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < words;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        a.reach0[e] = a.candb[e];
        a.active[e] = a.srcb[e];
    }
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        a.controller[s] = kInvalid32;
        a.reach_step[s] = cand[s] ? 0u : kInvalid32;
    }
}

// D' = (valid && !reachable) || unsafe, from the previous iteration's set.
__global__ void k_fused_dp(GridInfo g, FusedFixArgs a) {
    const FixControl* fc = a.fc;
    if (fc->stop) return;
    const uint64_t* rprev = (fc->iter & 1) ? a.reach1 : a.reach0;
    const uint64_t words = g.rows * g.W;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < words;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        a.dp[e] = (a.validb[e] & ~rprev[e]) | a.unsafeb[e];
}

template <int W>
__device__ __forceinline__ uint64_t extract_bits(const uint64_t (&F)[W], uint32_t lx, uint32_t hx) {
    const uint32_t wi = lx >> 6, sh = lx & 63u, len = hx - lx + 1;
    uint64_t lo = 0, hi = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        if (static_cast<uint32_t>(w) == wi) lo = F[w];
        if (static_cast<uint32_t>(w) == wi + 1) hi = F[w];
    }
    const uint64_t v = sh ? ((lo >> sh) | (hi << (64 - sh))) : lo;
    const uint64_t mask = len >= 64 ? ~0ull : ((1ull << len) - 1);
    return v & mask;
}

// acc |= F shifted so that bit i of the result is bit i + d of F (|d| < 64).
template <int W>
__device__ __forceinline__ void or_shifted(const uint64_t (&F)[W], int d, uint64_t (&acc)[W]) {
    if (d >= 0) {
        const uint32_t r = static_cast<uint32_t>(d);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            uint64_t v = F[w] >> r;
            if (w + 1 < W && r) v |= F[w + 1] << (64 - r);
            acc[w] |= v;
        }
    } else {
        const uint32_t r = static_cast<uint32_t>(-d);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            uint64_t v = F[w] << r;
            if (w > 0) v |= F[w - 1] >> (64 - r);
            acc[w] |= v;
        }
    }
}

// One block per (theta, v) slice, all (x, y) states of the slice.
//
// Inputs are visited omega-column by omega-column (j = ja + ma * jw).  For one
// column every input shares the theta range of its box, so the block first ORs
// the D' rows over that theta range for every v row the column can reach
// (Ez, shared memory).  Then each warp takes one acceleration ja: E[y] = OR of
// Ez over the v range of input j, F[i1] = OR of E over the y range of row i1,
// and the x test runs 64 states at a time: the x boxes of a plane fall into a
// few classes (lo - i0, hi - i0) = (a, b), and a state in class c is blocked
// when F has a bit in [i0 + a, i0 + b], i.e. when bit i0 of
// OR_{d=a..b} (F >> d) is set.  A plane with more than kClassMax classes uses
// the per-state test.  The block then resolves the column in input order, so
// every state records the lowest satisfied input.
template <int W, bool NV>
__global__ void __launch_bounds__(kFusedWarps * 32) k_sat_fused(GridInfo g, FusedFixArgs a) {
    extern __shared__ __align__(16) uint64_t smem[];
    __shared__ int s_wlo, s_whi;
    const FixControl* fc = a.fc;
    if (fc->stop) return;
    const uint32_t it = fc->iter + 1;
    const uint64_t* __restrict__ rprev = (fc->iter & 1) ? a.reach1 : a.reach0;
    uint64_t* __restrict__ rnext = (fc->iter & 1) ? a.reach0 : a.reach1;
    const uint32_t n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], ma = g.ma;
    const uint32_t nw = n1 * W;
    const uint32_t slice = blockIdx.x;
    const uint32_t i2 = slice % n2, i3 = slice / n2;
    const uint64_t wbase = static_cast<uint64_t>(slice) * nw;
    const uint32_t tid = threadIdx.x, bd = blockDim.x;
    const uint32_t warp = tid >> 5, lane = tid & 31;
    const uint32_t nv = NV ? 2u : 1u;

    uint64_t* act = smem;
    uint64_t* fnd = act + nw;
    uint64_t* Ez = fnd + nw;                       // ez_rows * nw (+ the same for valid)
    uint64_t* sat = Ez + a.ez_rows * nw * nv;      // ma * nw
    uint64_t* mine = sat + ma * nw + warp * (nw * nv + a.cls_words);
    uint64_t* E = mine;                            // nw (+ nw valid)
    uint64_t* cls = mine + nw * nv;                // class record of the warp's plane

    int any = 0;
    for (uint32_t e = tid; e < nw; e += bd) {
        const uint64_t v = a.active[wbase + e];
        act[e] = v;
        fnd[e] = 0;
        any |= (v != 0);
    }
    if (tid == 0) {
        int lo = 1 << 30, hi = -1;
        for (uint32_t ja = 0; ja < ma; ++ja) {
            const uint32_t we = a.wt[i3 * ma + ja];
            if (we == kReject) continue;
            lo = min(lo, static_cast<int>(lo16(we)));
            hi = max(hi, static_cast<int>(hi16(we)));
        }
        s_wlo = lo;
        s_whi = hi;
    }
    any = __syncthreads_or(any);
    const int wlo = s_wlo, whi = s_whi;
    if (!any || whi < wlo) {
        for (uint32_t e = tid; e < nw; e += bd) rnext[wbase + e] = rprev[wbase + e];
        return;
    }
    const uint32_t nwu = static_cast<uint32_t>(whi - wlo + 1);
    unsigned long long ntest = 0, nplane = 0;
    for (uint32_t jw = 0; jw < g.mw; ++jw) {
        const uint32_t ze = a.zt[i2 * g.mw + jw];
        const uint32_t lz = lo16(ze), hz = hi16(ze);
        for (uint32_t e = tid; e < nwu * nw; e += bd) {
            const uint32_t wr = e / nw, rem = e - wr * nw;
            const uint32_t y = rem / W, w = rem - y * W;
            const uint64_t wv = static_cast<uint64_t>(wlo) + wr;
            uint64_t acc = 0, accv = 0;
            uint32_t z = lz;
            for (;;) {
                const uint64_t r = y + static_cast<uint64_t>(n1) * (z + static_cast<uint64_t>(n2) * wv);
                acc |= __ldg(a.dp + r * W + w);
                if (NV) accv |= __ldg(a.validb + r * W + w);
                if (z == hz) break;
                z = (z + 1 == n2) ? 0 : z + 1;
            }
            Ez[e] = acc;
            if (NV) Ez[nwu * nw + e] = accv;
        }
        __syncthreads();
        for (uint32_t ja = warp; ja < ma; ja += kFusedWarps) {
            const uint32_t j = ja + ma * jw;
            uint64_t* Sj = sat + ja * nw;
            const uint32_t we = a.wt[i3 * ma + ja];
            if (we == kReject) {
                for (uint32_t e = lane; e < nw; e += 32) Sj[e] = 0;
                continue;
            }
            nplane += (lane == 0);
            const uint32_t lw = lo16(we) - wlo, hw = hi16(we) - wlo;
            const uint64_t plane = (static_cast<uint64_t>(i2) * g.n[3] + i3) * g.M + j;
            for (uint32_t e = lane; e < a.cls_words; e += 32) cls[e] = __ldg(a.xcls + plane * a.cls_words + e);
            for (uint32_t e = lane; e < nw; e += 32) {
                uint64_t acc = 0, accv = 0;
                for (uint32_t wr = lw; wr <= hw; ++wr) {
                    acc |= Ez[wr * nw + e];
                    if (NV) accv |= Ez[(nwu + wr) * nw + e];
                }
                E[e] = acc;
                if (NV) E[nw + e] = accv;
            }
            __syncwarp();
            const uint64_t h0 = cls[0], h1 = cls[1];
            const uint32_t ncls = static_cast<uint32_t>(h0 & 0xFFu);
            uint64_t okm[W];
#pragma unroll
            for (int w = 0; w < W; ++w) okm[w] = 0;
            if (ncls != 0xFFu) {
                for (uint32_t c = 0; c < ncls; ++c) {
#pragma unroll
                    for (int w = 0; w < W; ++w) okm[w] |= cls[2 + c * W + w];
                }
            }
            for (uint32_t i1 = lane; i1 < n1; i1 += 32) {
                uint64_t cm[W], sw[W];
                bool anyc = false;
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    cm[w] = act[i1 * W + w] & ~fnd[i1 * W + w];
                    sw[w] = 0;
                    anyc |= cm[w] != 0;
                }
                const uint32_t ye = anyc ? __ldg(a.yt + plane * n1 + i1) : kReject;
                if (ye != kReject) {
#pragma unroll
                    for (int w = 0; w < W; ++w) ntest += __popcll(cm[w]);
                    uint64_t F[W], FV[W];
#pragma unroll
                    for (int w = 0; w < W; ++w) F[w] = FV[w] = 0;
                    for (uint32_t y = lo16(ye); y <= hi16(ye); ++y) {
#pragma unroll
                        for (int w = 0; w < W; ++w) {
                            F[w] |= E[y * W + w];
                            if (NV) FV[w] |= E[nw + y * W + w];
                        }
                    }
                    if (ncls != 0xFFu) {
                        uint64_t U[W], VA[W];
#pragma unroll
                        for (int w = 0; w < W; ++w) U[w] = VA[w] = 0;
                        for (uint32_t c = 0; c < ncls; ++c) {
                            const int ca = static_cast<int8_t>((h0 >> (8 * (c + 1))) & 0xFFu);
                            const int cb = static_cast<int8_t>((h1 >> (8 * c)) & 0xFFu);
                            uint64_t win[W], winv[W];
#pragma unroll
                            for (int w = 0; w < W; ++w) win[w] = winv[w] = 0;
                            for (int d = ca; d <= cb; ++d) {
                                or_shifted<W>(F, d, win);
                                if (NV) or_shifted<W>(FV, d, winv);
                            }
#pragma unroll
                            for (int w = 0; w < W; ++w) {
                                const uint64_t m = cls[2 + c * W + w];
                                U[w] |= win[w] & m;
                                VA[w] |= winv[w] & m;
                            }
                        }
#pragma unroll
                        for (int w = 0; w < W; ++w) sw[w] = cm[w] & okm[w] & ~U[w] & (NV ? VA[w] : ~0ull);
                    } else {
                        const uint32_t* xrow = a.xt + plane * n0;
#pragma unroll
                        for (int w = 0; w < W; ++w) {
                            uint64_t m = cm[w];
                            while (m) {
                                const uint32_t b = __ffsll(static_cast<long long>(m)) - 1;
                                m &= m - 1;
                                const uint32_t xe = __ldg(xrow + w * 64 + b);
                                if (xe == kReject) continue;
                                const uint32_t lx = lo16(xe), hx = hi16(xe);
                                bool ok = extract_bits<W>(F, lx, hx) == 0;
                                if (NV) ok = ok && extract_bits<W>(FV, lx, hx) != 0;
                                if (ok) sw[w] |= 1ull << b;
                            }
                        }
                    }
                }
#pragma unroll
                for (int w = 0; w < W; ++w) Sj[i1 * W + w] = sw[w];
            }
        }
        __syncthreads();
        // Resolve the column in input order: the lowest satisfied input wins.
        int left = 0;
        for (uint32_t e = tid; e < nw; e += bd) {
            uint64_t f = fnd[e];
            uint64_t open = act[e] & ~f;
            const uint64_t srow = (static_cast<uint64_t>(slice) * n1 + e / W) * n0 + (e % W) * 64;
            for (uint32_t ja = 0; ja < ma && open; ++ja) {
                const uint64_t nb = sat[ja * nw + e] & open;
                if (!nb) continue;
                open &= ~nb;
                f |= nb;
                uint64_t m = nb;
                while (m) {
                    const uint32_t b = __ffsll(static_cast<long long>(m)) - 1;
                    m &= m - 1;
                    a.controller[srow + b] = ja + ma * jw;
                }
            }
            fnd[e] = f;
            left |= (open != 0);
        }
        if (!__syncthreads_or(left)) break;
    }
    unsigned long long nr = 0, nc = 0;
    for (uint32_t e = tid; e < nw; e += bd) {
        const uint64_t f = fnd[e];
        const uint64_t gi = wbase + e;
        const uint64_t rp = rprev[gi];
        rnext[gi] = rp | f;
        if (f) {
            a.active[gi] = act[e] & ~f;
            const uint64_t c = a.candb[gi];
            nr += __popcll(f & ~rp);
            nc += __popcll(f & c);
            uint64_t m = f & ~c;
            const uint64_t sbase = (static_cast<uint64_t>(slice) * n1 + e / W) * n0 + (e % W) * 64;
            while (m) {
                const uint32_t b = __ffsll(static_cast<long long>(m)) - 1;
                m &= m - 1;
                a.reach_step[sbase + b] = it;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        nr += __shfl_down_sync(0xFFFFFFFFu, nr, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
        ntest += __shfl_down_sync(0xFFFFFFFFu, ntest, off);
        nplane += __shfl_down_sync(0xFFFFFFFFu, nplane, off);
    }
    if ((tid & 31) == 0) {
        unsigned long long* row = a.stats + kStatsCols * it;
        if (nr) atomicAdd(row, nr);
        if (nc) atomicAdd(row + 1, nc);
        if (ntest) atomicAdd(row + 2, ntest);
        if (nplane) atomicAdd(row + 3, nplane);
    }
}

template <int W, bool NV>
cudaError_t launch_sat_fused_t(const GridInfo& g, const FusedFixArgs& a, size_t sm, cudaStream_t st) {
    // The opt-in above 48 KB is a per-device function attribute: set it once per device.
    static bool configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !configured[dev]) {
        e = cudaFuncSetAttribute(k_sat_fused<W, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kFusedSmemMax));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev] = true;
    }
    k_sat_fused<W, NV><<<g.slices, kFusedWarps * 32, sm, st>>>(g, a);
    return cudaGetLastError();
}

}  // namespace

size_t fused_smem_bytes(const GridInfo& g, uint32_t ez_rows, uint32_t cls_words, int need_valid) {
    const size_t nw = static_cast<size_t>(g.n[1]) * g.W;
    const size_t nv = need_valid ? 2 : 1;
    return 8 * (2 * nw + ez_rows * nw * nv + g.ma * nw + kFusedWarps * (nw * nv + cls_words));
}

namespace {
}  // namespace

cudaError_t launch_prefix4(const GridInfo& g, int mode, const uint8_t* a, const uint8_t* b, int32_t* table,
                           const FixControl* ctl, cudaStream_t st) {
    k_prefix_x<<<blocks_for(g.rows * 32, 256), 256, 0, st>>>(g, mode, a, b, table, ctl);
    for (int dim = 1; dim <= 3; ++dim) {
        const int d1 = (dim == 1) ? 2 : 1;
        const int d2 = (dim == 3) ? 2 : 3;
        const uint64_t lines = static_cast<uint64_t>(g.n[0]) * g.n[d1] * g.n[d2];
        k_prefix_axis<<<blocks_for(lines, 256), 256, 0, st>>>(g, dim, table, ctl);
    }
    return cudaGetLastError();
}

cudaError_t launch_stored_init(const GridInfo& g, const StoredFixArgs& a, cudaStream_t st) {
    k_stored_init<<<blocks_for(g.S, 256), 256, 0, st>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_stored_iteration(const GridInfo& g, const StoredFixArgs& a, cudaStream_t st, uint32_t* launches,
                                    cudaEvent_t* ev) {
    if (ev) cudaEventRecord(ev[0], st);
    cudaError_t e = launch_prefix4(g, 1, a.valid, a.reach, a.pd, a.fc, st);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[1], st);
    k_sat_stored<<<blocks_for(a.S_pad / 2, 256), 256, 0, st>>>(g, a);
    if (ev) cudaEventRecord(ev[2], st);
    k_control<<<1, 1, 0, st>>>(a.fc, a.stats, a.cond, a.use_cond);
    if (launches) *launches += 6;
    return cudaGetLastError();
}

cudaError_t launch_fused_init(const GridInfo& g, const FusedFixArgs& a, const uint8_t* cand, cudaStream_t st) {
    k_fused_init<<<blocks_for(g.S, 256), 256, 0, st>>>(g, a, cand);
    return cudaGetLastError();
}

cudaError_t launch_fused_iteration(const GridInfo& g, const FusedFixArgs& a, cudaStream_t st, uint32_t* launches,
                                   cudaEvent_t* ev) {
    if (ev) cudaEventRecord(ev[0], st);
    k_fused_dp<<<blocks_for(g.rows * g.W, 256), 256, 0, st>>>(g, a);
    if (ev) cudaEventRecord(ev[1], st);
    const size_t sm = fused_smem_bytes(g, a.ez_rows, a.cls_words, a.need_valid);
    cudaError_t err;
    if (a.need_valid) {
        switch (g.W) {
            case 1: err = launch_sat_fused_t<1, true>(g, a, sm, st); break;
            case 2: err = launch_sat_fused_t<2, true>(g, a, sm, st); break;
            case 3: err = launch_sat_fused_t<3, true>(g, a, sm, st); break;
            default: err = launch_sat_fused_t<4, true>(g, a, sm, st); break;
        }
    } else {
        switch (g.W) {
            case 1: err = launch_sat_fused_t<1, false>(g, a, sm, st); break;
            case 2: err = launch_sat_fused_t<2, false>(g, a, sm, st); break;
            case 3: err = launch_sat_fused_t<3, false>(g, a, sm, st); break;
            default: err = launch_sat_fused_t<4, false>(g, a, sm, st); break;
        }
    }
    if (err != cudaSuccess) return err;
    if (ev) cudaEventRecord(ev[2], st);
    k_control<<<1, 1, 0, st>>>(a.fc, a.stats, a.cond, a.use_cond);
    if (launches) *launches += 3;
    return cudaGetLastError();
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
