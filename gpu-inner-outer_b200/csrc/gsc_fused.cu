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
#include "gsc_kernels.cuh"

namespace gsc_b200 {

namespace {

inline unsigned int blocks_for(uint64_t n, int threads) {
    uint64_t b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return static_cast<unsigned int>(b);
}

// Bits [lx, hx] of the row F (hx - lx < 32), in the low bits.
template <int W>
__device__ __forceinline__ bword extract_bits(const bword (&F)[W], uint32_t lx, uint32_t hx) {
    const uint32_t wi = lx / kBits, sh = lx % kBits, len = hx - lx + 1;
    bword lo = 0, hi = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        if (static_cast<uint32_t>(w) == wi) lo = F[w];
        if (static_cast<uint32_t>(w) == wi + 1) hi = F[w];
    }
    const bword v = __funnelshift_r(lo, hi, sh);
    return len >= kBits ? v : (v & ((bword(1) << len) - 1));
}

// acc |= F shifted so that bit i of the result is bit i + d of F (|d| < 32):
// one funnel shift per word.
template <int W>
__device__ __forceinline__ void or_shifted(const bword (&F)[W], int d, bword (&acc)[W]) {
    if (d >= 0) {
#pragma unroll
        for (int w = 0; w < W; ++w) acc[w] |= __funnelshift_r(F[w], (w + 1 < W) ? F[w + 1] : 0u, d);
    } else {
#pragma unroll
        for (int w = 0; w < W; ++w) acc[w] |= __funnelshift_l((w > 0) ? F[w - 1] : 0u, F[w], -d);
    }
}

__device__ __forceinline__ int hdr_byte(const bword* rec, int k) {
    return static_cast<int8_t>((rec[k >> 2] >> (8 * (k & 3))) & 0xFFu);
}

__global__ void k_fused_init(GridInfo g, FusedFixArgs a, const uint8_t* __restrict__ cand) {
    const uint64_t words = g.rows * g.W;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < words;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const bword c = a.candb[e];
        a.reach0[e] = c;
        a.active[e] = a.srcb[e];
        a.hit[e] = 0;
        a.dp[e] = (a.validb[e] & ~c) | a.unsafeb[e];
    }
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < g.S;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        a.controller[s] = kInvalid32;
        a.reach_step[s] = cand[s] ? 0u : kInvalid32;
        a.best[s] = kInvalid32;
    }
}

// (theta, v)-dilated copies of a bit-sliced set: for every theta width k in
// d.kval and v width l in d.lval, out[combo][y][z][v] = OR of src over
// theta cells z .. z+k-1 (wrapped) and v cells v .. v+l-1 (entries whose v
// window leaves the grid are never read and are left 0).  One thread per
// word position; the theta ORs are extended incrementally.
__global__ void k_dilate(GridInfo g, const bword* __restrict__ src, bword* __restrict__ dst, DilateArgs d,
                         const FixControl* fc) {
    if (fc && fc->stop) return;
    const uint32_t n1 = g.n[1], n2 = g.n[2], n3 = g.n[3], W = g.W;
    const uint32_t pos = static_cast<uint32_t>(g.rows * W);
    const uint32_t kmax = d.kval[d.nk - 1];
    uint32_t lmax = d.lval[d.nl - 1];
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pos; p += gridDim.x * blockDim.x) {
        const uint32_t r = p / W, wd = p - r * W;
        const uint32_t y = r % n1, q = r / n1;
        const uint32_t z = q % n2, v = q / n2;
        const uint32_t lfit = min(lmax, n3 - v);   // v windows that stay inside the grid
        bword zor[kMaxDilate];
#pragma unroll
        for (uint32_t j = 0; j < kMaxDilate; ++j) zor[j] = 0;
        uint32_t ki = 0, zz = z;
        for (uint32_t i = 0; i < kmax; ++i) {
#pragma unroll
            for (uint32_t j = 0; j < kMaxDilate; ++j)
                if (j < lfit) zor[j] |= __ldg(src + (y + n1 * (zz + n2 * (v + j))) * W + wd);
            zz = (zz + 1 == n2) ? 0 : zz + 1;
            if (i + 1 == d.kval[ki]) {
                bword acc = 0;
                uint32_t li = 0;
#pragma unroll
                for (uint32_t j = 0; j < kMaxDilate; ++j) {
                    acc |= zor[j];
                    if (li < d.nl && j + 1 == d.lval[li]) {
                        dst[static_cast<uint64_t>(ki * d.nl + li) * pos + p] = (j < lfit) ? acc : 0u;
                        ++li;
                    }
                }
                ++ki;
            }
        }
    }
}

// The set-up plan (one block): which theta widths (wrapped lengths of the
// omega columns' theta boxes) and v widths (of the accelerations' v boxes)
// occur, numbered in increasing order, and the most representative
// accelerations of one omega column.
__global__ void __launch_bounds__(256) k_plan(GridInfo g, const uint32_t* __restrict__ zt,
                                              const uint32_t* __restrict__ wt, const uint8_t* __restrict__ xrep,
                                              const unsigned long long* __restrict__ counts,
                                              const unsigned int* __restrict__ flags, uint8_t* __restrict__ kidx,
                                              uint8_t* __restrict__ lidx, PlanRecord* __restrict__ out) {
    __shared__ uint32_t kbits[2048], lbits[2048];   // widths 1 .. 65535
    __shared__ uint32_t s_maxrep;
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
    if (tid == 0) s_maxrep = 1;
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
    const uint64_t columns = static_cast<uint64_t>(g.slices) * g.mw;
    uint32_t mr = 1;
    for (uint64_t c = tid; c < columns; c += blockDim.x) {
        uint32_t n = 0;
        for (uint32_t ja = 0; ja < g.ma; ++ja) n += xrep[c * g.ma + ja] == ja;
        mr = max(mr, n);
    }
    atomicMax(&s_maxrep, mr);
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
        out->max_reps = s_maxrep;
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

// One block per (theta, v) slice x omega column jw.
//  B. per representative acceleration (the lowest of each group of inputs
//     whose boxes coincide), E[y] = the (theta, v)-dilated D' row at the
//     input's box corner: one load per word;
//  C. each (representative, i1) item: F = OR of E over row i1's y range, then
//     the x test 32 states per word: the x boxes of a plane fall into a few
//     classes (lo - i0, hi - i0) = (a, b), and a state of class (a, b) is
//     blocked when F has a bit in [i0 + a, i0 + b], i.e. bit i0 of
//     OR_{d=a..b} (F >> d); a plane with more than kClassMax classes is tested
//     state by state;
//  D. per state, the lowest satisfied input of the column goes to best[]
//     (atomicMin, so the lowest over all columns wins) and the hit bit is set.
template <int W, bool NV>
__global__ void __launch_bounds__(kFusedWarps * 32) k_sat_col(GridInfo g, FusedFixArgs a) {
    extern __shared__ __align__(16) bword smem[];
    __shared__ uint32_t s_nrep;
    const FixControl* fc = a.fc;
    if (fc->stop) return;
    const uint32_t n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], ma = g.ma, mw = g.mw;
    const uint32_t nw = n1 * W;
    const uint32_t slice = blockIdx.x / mw, jw = blockIdx.x - slice * mw;
    const uint32_t i2 = slice % n2, i3 = slice / n2;
    const uint64_t wbase = static_cast<uint64_t>(slice) * nw;
    const uint32_t tid = threadIdx.x, bd = blockDim.x;
    const uint32_t lane = tid & 31;
    const uint32_t nv = NV ? 2u : 1u;
    const uint32_t cw = a.cls_words;
    const uint32_t mr = a.max_reps;
    const uint32_t pos = static_cast<uint32_t>(g.rows * W);

    bword* act = smem;
    bword* Eall = act + nw;                               // max_reps * nw * nv
    bword* sat = Eall + mr * nw * nv;                     // max_reps * nw
    bword* cls = sat + mr * nw;                           // max_reps * cw
    uint32_t* yts = cls + mr * cw;                        // max_reps * n1
    uint32_t* reps = yts + mr * n1;                       // ma: acceleration of each representative slot

    const uint64_t pcol = (static_cast<uint64_t>(i2) * g.n[3] + i3) * g.M + static_cast<uint64_t>(ma) * jw;
    int any = 0;
    for (uint32_t e = tid; e < nw; e += bd) {
        const bword v = a.active[wbase + e];
        act[e] = v;
        any |= (v != 0);
    }
    if (tid < 32) {
        // Representatives in increasing acceleration order (warp ballot).
        uint32_t n = 0;
        for (uint32_t base = 0; base < ma; base += 32) {
            const uint32_t ja = base + lane;
            const bool is_rep = ja < ma && a.xrep[pcol + ja] == ja && a.wt[i3 * ma + ja] != kReject;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, is_rep);
            if (is_rep) reps[n + __popc(m & ((1u << lane) - 1))] = ja;
            n += __popc(m);
        }
        if (lane == 0) s_nrep = n;
    }
    any = __syncthreads_or(any);
    const uint32_t nrep = s_nrep;
    if (!any || nrep == 0) return;
    if (tid == 0) atomicAdd(a.stats + kStatsCols * (fc->iter + 1) + 3, static_cast<unsigned long long>(nrep));

    // B. dilated D' rows at each representative's (theta, v) box corner.
    const uint32_t ze = a.zt[i2 * mw + jw];
    const uint32_t lz = lo16(ze), hz = hi16(ze);
    const uint32_t nz = (lz <= hz) ? hz - lz + 1 : n2 - lz + hz + 1;
    const uint32_t kslot = a.kidx[nz];
    for (uint32_t e = tid; e < nrep * nw; e += bd) {
        const uint32_t r = fdiv(e, g.magic_nw), rem = e - r * nw;
        const uint32_t y = rem / W, wd = rem - y * W;
        const uint32_t we = a.wt[i3 * ma + reps[r]];
        const uint32_t lw = lo16(we), nwb = hi16(we) - lw + 1;
        const uint64_t off = static_cast<uint64_t>(kslot * a.nl + a.lidx[nwb]) * pos +
                             (y + n1 * (lz + n2 * lw)) * W + wd;
        Eall[r * nw * nv + rem] = __ldg(a.dzw + off);
        if (NV) Eall[r * nw * nv + nw + rem] = __ldg(a.vzw + off);
    }
    for (uint32_t r = tid >> 5; r < nrep; r += bd >> 5) {
        const uint64_t pl = pcol + reps[r];
        for (uint32_t e = lane; e < cw; e += 32) cls[r * cw + e] = __ldg(a.xcls + pl * cw + e);
        for (uint32_t e = lane; e < n1; e += 32) yts[r * n1 + e] = __ldg(a.yt + pl * n1 + e);
    }
    __syncthreads();
    // C. the (representative, row) items.
    unsigned long long ntest = 0;
    for (uint32_t e = tid; e < nrep * n1; e += bd) {
        const uint32_t r = fdiv(e, g.magic_n1), i1 = e - r * n1;
        const uint32_t ja = reps[r];
        bword cm[W], sw[W];
        bword anyc = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            cm[w] = act[i1 * W + w];
            sw[w] = 0;
            anyc |= cm[w];
        }
        const uint32_t ye = yts[r * n1 + i1];
        if (anyc && ye != kReject) {
#pragma unroll
            for (int w = 0; w < W; ++w) ntest += __popc(cm[w]);
            const bword* E = Eall + r * nw * nv;
            bword F[W], FV[W];
#pragma unroll
            for (int w = 0; w < W; ++w) F[w] = FV[w] = 0;
            for (uint32_t y = lo16(ye); y <= hi16(ye); ++y) {
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    F[w] |= E[y * W + w];
                    if (NV) FV[w] |= E[nw + y * W + w];
                }
            }
            const bword* rec = cls + r * cw;
            const uint32_t ncls = rec[0] & 0xFFu;
            if (ncls != 0xFFu) {
                bword U[W], VA[W], OK[W];
#pragma unroll
                for (int w = 0; w < W; ++w) U[w] = VA[w] = OK[w] = 0;
                for (uint32_t c = 0; c < ncls; ++c) {
                    const int ca = hdr_byte(rec, 1 + c);
                    const int cb = hdr_byte(rec, 7 + c);
                    bword win[W], winv[W];
#pragma unroll
                    for (int w = 0; w < W; ++w) win[w] = winv[w] = 0;
                    for (int d = ca; d <= cb; ++d) {
                        or_shifted<W>(F, d, win);
                        if (NV) or_shifted<W>(FV, d, winv);
                    }
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const bword m = rec[4 + c * W + w];
                        OK[w] |= m;
                        U[w] |= win[w] & m;
                        if (NV) VA[w] |= winv[w] & m;
                    }
                }
#pragma unroll
                for (int w = 0; w < W; ++w) sw[w] = cm[w] & OK[w] & ~U[w] & (NV ? VA[w] : ~0u);
            } else {
                const uint32_t* xrow = a.xt + (pcol + ja) * n0;
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    bword m = cm[w];
                    while (m) {
                        const uint32_t b = __ffs(m) - 1;
                        m &= m - 1;
                        const uint32_t xe = __ldg(xrow + w * kBits + b);
                        if (xe == kReject) continue;
                        const uint32_t lx = lo16(xe), hx = hi16(xe);
                        bool ok = extract_bits<W>(F, lx, hx) == 0;
                        if (NV) ok = ok && extract_bits<W>(FV, lx, hx) != 0;
                        if (ok) sw[w] |= bword(1) << b;
                    }
                }
            }
        }
#pragma unroll
        for (int w = 0; w < W; ++w) sat[r * nw + i1 * W + w] = sw[w];
    }
    __syncthreads();
    // D. lowest satisfied input of the column per state -> best[] and hit
    // bits.  Representatives are in increasing order and each is the lowest
    // input of its group, so the first representative that satisfies a state
    // gives its lowest satisfied input of the column.
    for (uint32_t e = tid; e < nw; e += bd) {
        bword open = act[e], got = 0;
        const uint32_t y = e / W;
        const uint64_t srow = (static_cast<uint64_t>(slice) * n1 + y) * n0 + (e - y * W) * kBits;
        for (uint32_t r = 0; r < nrep && open; ++r) {
            const bword nb = sat[r * nw + e] & open;
            if (!nb) continue;
            open &= ~nb;
            got |= nb;
            const uint32_t j = reps[r] + ma * jw;
            bword m = nb;
            while (m) {
                const uint32_t b = __ffs(m) - 1;
                m &= m - 1;
                atomicMin(a.best + srow + b, j);
            }
        }
        if (got) atomicOr(a.hit + wbase + e, got);
    }
    for (int off = 16; off > 0; off >>= 1) ntest += __shfl_down_sync(0xFFFFFFFFu, ntest, off);
    if ((tid & 31) == 0 && ntest) atomicAdd(a.stats + kStatsCols * (fc->iter + 1) + 2, ntest);
}

// Apply the iteration's hits, build next iteration's D', count, and let the
// last block to finish apply the stop rules (reachability.hpp:133-144).
__global__ void __launch_bounds__(256) k_fused_finalize(GridInfo g, FusedFixArgs a) {
    FixControl* fc = a.fc;
    if (fc->stop) {
        // Already stopped (e.g. max_iterations == 0): the graph loop must still end.
        if (a.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
        return;
    }
    const uint32_t it = fc->iter + 1;
    const bword* __restrict__ rprev = (fc->iter & 1) ? a.reach1 : a.reach0;
    bword* __restrict__ rnext = (fc->iter & 1) ? a.reach0 : a.reach1;
    const uint64_t words = g.rows * g.W;
    unsigned long long nr = 0, nc = 0;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < words;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const bword rp = rprev[e];
        const bword h = a.hit[e];
        const bword rn = rp | h;
        rnext[e] = rn;
        a.dp[e] = (a.validb[e] & ~rn) | a.unsafeb[e];
        if (h) {
            a.hit[e] = 0;
            a.active[e] &= ~h;
            const bword c = a.candb[e];
            nr += __popc(h & ~rp);
            nc += __popc(h & c);
            const uint64_t r = e / g.W;
            const uint64_t sbase = r * g.n[0] + (e - r * g.W) * kBits;
            bword m = h;
            while (m) {
                const uint32_t b = __ffs(m) - 1;
                m &= m - 1;
                const uint64_t s = sbase + b;
                a.controller[s] = a.best[s];
                a.best[s] = kInvalid32;
                if (!((c >> b) & 1u)) a.reach_step[s] = it;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        nr += __shfl_down_sync(0xFFFFFFFFu, nr, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
    }
    unsigned long long* row = a.stats + kStatsCols * it;
    if ((threadIdx.x & 31) == 0) {
        if (nr) atomicAdd(row, nr);
        if (nc) atomicAdd(row + 1, nc);
    }
    // Last block to finish: every block's counters are in (device-scope
    // atomics, then a fence before taking a ticket).
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&fc->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    if (threadIdx.x == 0) {
        __threadfence();
        fc->ticket = 0;
        const unsigned long long tnr = atomicAdd(row, 0ull);
        const unsigned long long tnc = atomicAdd(row + 1, 0ull);
        fc->certified += tnc;
        fc->reachable += tnr;
        fc->iter = it;
        if (fc->certified == fc->candidate_count) {
            fc->converged = 1;
            fc->message = 1;
            fc->stop = 1;
        } else if (tnr == 0 && tnc == 0) {
            fc->message = 2;
            fc->stop = 1;
        } else if (it >= fc->max_iterations || it + 1 >= fc->stats_cap) {
            fc->message = 3;
            fc->stop = 1;
        }
        if (a.use_cond) cudaGraphSetConditional(a.cond, fc->stop ? 0u : 1u);
    }
}

template <int W, bool NV>
cudaError_t launch_sat_col_t(const GridInfo& g, const FusedFixArgs& a, size_t sm, cudaStream_t st) {
    // Opting in above 48 KB of shared memory is a per-device function attribute.
    static bool configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !configured[dev]) {
        e = cudaFuncSetAttribute(k_sat_col<W, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kFusedSmemMax));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev] = true;
    }
    k_sat_col<W, NV><<<g.slices * g.mw, kFusedWarps * 32, sm, st>>>(g, a);
    return cudaGetLastError();
}

}  // namespace

size_t fused_smem_bytes(const GridInfo& g, uint32_t cls_words, int need_valid, uint32_t max_reps) {
    const size_t nw = static_cast<size_t>(g.n[1]) * g.W;
    const size_t nv = need_valid ? 2 : 1;
    const size_t mr = max_reps;
    const size_t words = nw + mr * nw * nv + mr * nw + mr * cls_words + mr * g.n[1] + static_cast<size_t>(g.ma);
    return sizeof(bword) * words;
}

cudaError_t launch_plan(const GridInfo& g, const uint32_t* zt, const uint32_t* wt, const uint8_t* xrep,
                        const unsigned long long* counts, const unsigned int* flags, uint8_t* kidx, uint8_t* lidx,
                        PlanRecord* out, cudaStream_t st) {
    if (xrep && (g.n[2] > 65535 || g.n[3] > 65535)) return cudaErrorInvalidValue;
    k_plan<<<1, 256, 0, st>>>(g, zt, wt, xrep, counts, flags, kidx, lidx, out);
    return cudaGetLastError();
}

cudaError_t launch_dilate(const GridInfo& g, const bword* src, bword* dst, const DilateArgs& d, const FixControl* fc,
                          cudaStream_t st) {
    const uint64_t pos = g.rows * g.W;
    uint64_t b = (pos + 255) / 256;
    if (b > 8192) b = 8192;
    k_dilate<<<static_cast<unsigned int>(b ? b : 1), 256, 0, st>>>(g, src, dst, d, fc);
    return cudaGetLastError();
}

cudaError_t launch_fused_init(const GridInfo& g, const FusedFixArgs& a, const uint8_t* cand, cudaStream_t st) {
    k_fused_init<<<blocks_for(g.S, 256), 256, 0, st>>>(g, a, cand);
    return cudaGetLastError();
}

cudaError_t launch_fused_iteration(const GridInfo& g, const FusedFixArgs& a, cudaStream_t st, uint32_t* launches,
                                   cudaEvent_t* ev) {
    if (ev) cudaEventRecord(ev[0], st);
    cudaError_t derr = launch_dilate(g, a.dp, a.dzw, a.dil, a.fc, st);
    if (derr != cudaSuccess) return derr;
    if (ev) cudaEventRecord(ev[1], st);
    const size_t sm = fused_smem_bytes(g, a.cls_words, a.need_valid, a.max_reps);
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
    if (ev) cudaEventRecord(ev[2], st);
    const uint64_t words = g.rows * g.W;
    uint64_t fb = (words + 255) / 256;
    if (fb > 4096) fb = 4096;
    k_fused_finalize<<<static_cast<unsigned int>(fb ? fb : 1), 256, 0, st>>>(g, a);
    if (launches) *launches += 3;
    return cudaGetLastError();
}

}  // namespace gsc_b200
