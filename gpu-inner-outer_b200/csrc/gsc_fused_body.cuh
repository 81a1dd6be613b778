// gsc_fused_body.cuh -- device bodies of the fused fixpoint, shared by the
// one-problem kernels (gsc_fused.cu) and the batched kernels (gsc_batch.cu),
// so that a problem computes the same bits alone and inside a batch.
//
// Semantics are those of reachability.hpp:53-153 (Jacobi update, lowest
// satisfied input, reach_step = iteration, stop rules in the reference's
// order).
#pragma once

#include "gsc_kernels.cuh"

namespace gsc_b200 {
namespace fused {

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

// Initial sets of word e: reachable = candidate, active = valid && safe
// source, D' = (valid && !candidate) || unsafe.
__device__ __forceinline__ void init_word(const FusedFixArgs& a, uint64_t e) {
    const bword c = a.candb[e];
    a.reach0[e] = c;
    a.active[e] = a.srcb[e];
    a.hit[e] = 0;
    a.dp[e] = (a.validb[e] & ~c) | a.unsafeb[e];
}

__device__ __forceinline__ void init_state(const FusedFixArgs& a, const uint8_t* cand, uint64_t s) {
    a.controller[s] = kInvalid32;
    a.reach_step[s] = cand[s] ? 0u : kInvalid32;
    a.best[s] = kInvalid32;
}

// FixControl at the start of a solve (counts: [0] valid, [1] candidates).
__device__ __forceinline__ void init_control(FixControl* fc, uint32_t max_iterations, uint32_t stats_cap,
                                             const unsigned long long* counts) {
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

// (theta, v)-dilated copies of a bit-sliced set at word position p: for
// every theta width k in d.kval and v width l in d.lval, out[combo][y][z][v]
// = OR of src over theta cells z .. z+k-1 (wrapped) and v cells v .. v+l-1
// (entries whose v window leaves the grid are never read and are left 0).
// The theta ORs are extended incrementally.
// With `lost` (the rows that lost a D' cell since the last dilation) the
// position is left as it is when no row of its widest window did.
__device__ __forceinline__ void dilate_position(const GridInfo& g, const bword* __restrict__ src,
                                                bword* __restrict__ dst, const DilateArgs& d, uint32_t p,
                                                const uint32_t* __restrict__ lost) {
    const uint32_t n1 = g.n[1], n2 = g.n[2], n3 = g.n[3], W = g.W;
    const uint32_t pos = static_cast<uint32_t>(g.rows * W);
    const uint32_t kmax = d.kval[d.nk - 1];
    const uint32_t lmax = d.lval[d.nl - 1];
    const uint32_t r = p / W, wd = p - r * W;
    const uint32_t y = r % n1, q = r / n1;
    const uint32_t z = q % n2, v = q / n2;
    const uint32_t lfit = min(lmax, n3 - v);   // v windows that stay inside the grid
    if (lost) {
        // Every bit of the window is read (no early exit), so the loads of
        // several theta cells are in flight together.
        uint32_t hit = 0, zz = z;
#pragma unroll 4
        for (uint32_t i = 0; i < kmax; ++i) {
#pragma unroll
            for (uint32_t j = 0; j < kMaxDilate; ++j) {
                if (j < lfit) {
                    const uint32_t rr = y + n1 * (zz + n2 * (v + j));
                    hit |= (lost[rr >> 5] >> (rr & 31)) & 1u;
                }
            }
            zz = (zz + 1 == n2) ? 0 : zz + 1;
        }
        if (!hit) return;
    }
    bword zor[kMaxDilate];
#pragma unroll
    for (uint32_t j = 0; j < kMaxDilate; ++j) zor[j] = 0;
    uint32_t ki = 0, zz = z;
#pragma unroll 2
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


// The group that runs one satisfaction task: the whole block, or one warp
// (WARP), with its barrier and its barrier-with-OR.
template <bool WARP>
__device__ __forceinline__ void group_sync() {
    if (WARP)
        __syncwarp();
    else
        __syncthreads();
}

template <bool WARP>
__device__ __forceinline__ int group_sync_or(int p) {
    if (WARP) {
        __syncwarp();
        return __any_sync(0xFFFFFFFFu, p);
    }
    return __syncthreads_or(p);
}

// One (theta, v) slice x omega column jw (task = slice * mw + jw) of the
// satisfaction test, by the whole block:
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
// WMAX: register words per row; EXACTW: g.W == WMAX (else g.W <= WMAX at run
// time).  NVMODE: 0 / 1 = validity test off / on, 2 = a.need_valid decides.
// WARP: the task is one warp's (its own smem and s_meta), else the block's.
// Every early return is taken by the whole group.
constexpr unsigned long long kIncrementalRows = 16;

template <int WMAX, bool EXACTW, int NVMODE, bool WARP = false>
__device__ __forceinline__ void sat_col_task(const GridInfo& g, const FusedFixArgs& a, uint32_t task,
                                             bword* smem, uint32_t* s_meta) {
    const FixControl* fc = a.fc;
    const uint32_t W = EXACTW ? static_cast<uint32_t>(WMAX) : g.W;
    const bool NV = NVMODE == 2 ? (a.need_valid != 0) : (NVMODE == 1);
    const uint32_t n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], ma = g.ma, mw = g.mw;
    const uint32_t nw = n1 * W;
    const uint32_t slice = task / mw, jw = task - slice * mw;
    const uint32_t i2 = slice % n2, i3 = slice / n2;
    const uint64_t wbase = static_cast<uint64_t>(slice) * nw;
    const uint32_t tid = WARP ? (threadIdx.x & 31u) : threadIdx.x;
    const uint32_t bd = WARP ? 32u : blockDim.x;
    const uint32_t lane = tid & 31;
    const uint32_t nv = NV ? 2u : 1u;
    const uint32_t cw = a.cls_words;
    const uint32_t mr = a.max_reps;

    bword* act = smem;
    bword* Eall = act + nw;                               // max_reps * nw * nv
    bword* sat = Eall + mr * nw * nv;                     // max_reps * nw
    bword* cls = sat + mr * nw;                           // max_reps * cw
    uint32_t* yts = cls + mr * cw;                        // max_reps * n1
    uint32_t* reps = yts + mr * n1;                       // ma: acceleration of each representative slot
    uint32_t* repw = reps + ma;                           // ma: its v window
    uint32_t* repo = repw + ma;                           // ma: its part of the dilated rows' offset
    uint32_t* rowchg = repo + ma;                         // max_reps * W1: y rows of a window that lost a cell
    const uint32_t W1 = (n1 + 31) / 32;

    const uint64_t pcol = (static_cast<uint64_t>(i2) * g.n[3] + i3) * g.M + static_cast<uint64_t>(ma) * jw;
    // A. One round of loads that depend on the task alone: the active rows
    // (two per thread before either is stored), the representatives in
    // increasing acceleration order (warp ballot) with their v windows and
    // offset parts, the omega column's theta window and offset part, and
    // the control record (s_meta: [0] representatives, [1] theta window,
    // [2] offset part, [3] iteration | incremental << 31, or all ones once
    // stopped).
    int any = 0;
    for (uint32_t e0 = tid; e0 < nw; e0 += 2 * bd) {
        const uint32_t e1 = e0 + bd;
        const bword v0 = a.active[wbase + e0];
        const bword v1 = e1 < nw ? a.active[wbase + e1] : 0u;
        act[e0] = v0;
        if (e1 < nw) act[e1] = v1;
        any |= (v0 | v1) != 0;
    }
    if (tid < 32) {
        uint32_t n = 0;
        for (uint32_t base = 0; base < ma; base += 32) {
            const uint32_t ja = base + lane;
            uint32_t we = kReject, ov = 0;
            bool is_rep = false;
            if (ja < ma) {
                we = a.wt[i3 * ma + ja];
                ov = a.offv[i3 * ma + ja];
                is_rep = a.xrep[pcol + ja] == ja && we != kReject;
            }
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, is_rep);
            if (is_rep) {
                const uint32_t k = n + __popc(m & ((1u << lane) - 1));
                reps[k] = ja;
                repw[k] = we;
                repo[k] = ov;
            }
            n += __popc(m);
        }
        if (lane == 0) s_meta[0] = n;
    }
    if (tid == (bd > 32 ? 32u : 0u)) {
        // After the first iteration, every active state failed every input
        // in the previous one, and D' only loses cells, so a state can newly
        // pass only if its box holds a cell that left D' in the previous
        // iteration.  When that iteration added few states (at most one per
        // kIncrementalRows x-rows; a new state touches the items of about
        // that many rows), the iteration runs incrementally (phase B).
        const uint32_t stop = fc->stop, it = fc->iter, last = fc->last_new;
        const bool inc = it > 0 && static_cast<unsigned long long>(last) * kIncrementalRows <= g.rows;
        s_meta[1] = a.zt[i2 * mw + jw];
        s_meta[2] = a.offz[i2 * mw + jw];
        s_meta[3] = stop ? 0xFFFFFFFFu : (it | (inc ? 0x80000000u : 0u));
    }
    any = group_sync_or<WARP>(any);
    const uint32_t nrep = s_meta[0], ctl = s_meta[3];
    if (ctl == 0xFFFFFFFFu || !any || nrep == 0) return;
    const uint32_t it = ctl & 0x7FFFFFFFu;
    const bool incremental = (ctl >> 31) != 0;
    const uint32_t ze = s_meta[1], offz = s_meta[2];
    const uint32_t lz = lo16(ze), hz = hi16(ze);
    const uint32_t nz = (lz <= hz) ? hz - lz + 1 : n2 - lz + hz + 1;

    // B. The dilated D' (and valid) rows at each representative's (theta, v)
    // box corner, its class records and y tables, copied asynchronously into
    // shared memory, all in flight together.  In an incremental iteration
    // the rows of each representative's (theta, v) window that lost a cell
    // (rowlost, from the finalize kernel) are gathered first: a block with
    // none stages nothing and skips, and a (representative, row) item whose
    // y range has none is skipped; their states still fail.
    auto stage = [&]() {
        for (uint32_t e = tid; e < nrep * nw; e += bd) {
            const uint32_t r = fdiv(e, g.magic_nw), rem = e - r * nw;
            const uint32_t off = offz + repo[r] + rem;
            cp_async4(Eall + r * nw * nv + rem, a.dzw + off);
            if (NV) cp_async4(Eall + r * nw * nv + nw + rem, a.vzw + off);
        }
        for (uint32_t r = tid >> 5; r < nrep; r += bd >> 5) {
            const uint64_t pl = pcol + reps[r];
            for (uint32_t e = lane; e < cw; e += 32) cp_async4(cls + r * cw + e, a.xcls + pl * cw + e);
            for (uint32_t e = lane; e < n1; e += 32) cp_async4(yts + r * n1 + e, a.yt + pl * n1 + e);
        }
    };
    if (!incremental) stage();
    int lost = 0;
    if (incremental) {
        const uint32_t* rl = a.rowlost + (it & 1) * a.rl_words;
        for (uint32_t e = tid; e < nrep * W1; e += bd) {
            const uint32_t r = e / W1, yw = e - r * W1;
            const uint32_t we = repw[r];
            uint32_t m = 0, z = lz;
            for (uint32_t i = 0; i < nz; ++i) {
                for (uint32_t v = lo16(we); v <= hi16(we); ++v) {
                    const uint32_t bit = n1 * (z + n2 * v) + yw * 32;
                    m |= __funnelshift_r(rl[bit >> 5], rl[(bit >> 5) + 1], bit & 31);
                }
                z = (z + 1 == n2) ? 0 : z + 1;
            }
            if (yw == W1 - 1 && (n1 & 31)) m &= (1u << (n1 & 31)) - 1;
            rowchg[r * W1 + yw] = m;
            lost |= m != 0;
        }
    }
    if (incremental) {
        if (!group_sync_or<WARP>(lost)) return;
        stage();
    }
    cp_async_wait_all();
    group_sync<WARP>();
    if (tid == 0) atomicAdd(a.stats + kStatsCols * (it + 1) + 3, static_cast<unsigned long long>(nrep));
    // C. the (representative, row) items.
    unsigned long long ntest = 0;
    for (uint32_t e = tid; e < nrep * n1; e += bd) {
        const uint32_t r = fdiv(e, g.magic_n1), i1 = e - r * n1;
        const uint32_t ja = reps[r];
        bword cm[WMAX], sw[WMAX];
        bword anyc = 0;
#pragma unroll
        for (int w = 0; w < WMAX; ++w) {
            cm[w] = (EXACTW || static_cast<uint32_t>(w) < W) ? act[i1 * W + w] : 0u;
            sw[w] = 0;
            anyc |= cm[w];
        }
        const uint32_t ye = yts[r * n1 + i1];
        if (anyc && ye != kReject && incremental) {
            // Bits [lo, hi] of the representative's changed-row mask (fused
            // boxes span at most 32 rows): one funnel shift.
            const uint32_t lo = lo16(ye), hi = hi16(ye);
            const uint32_t* rc = rowchg + r * W1;
            const uint32_t wl = lo >> 5, wh = hi >> 5;
            const uint32_t bits = __funnelshift_r(rc[wl], wh != wl ? rc[wh] : 0u, lo & 31);
            const uint32_t len = hi - lo + 1;
            if (!(len >= 32 ? bits : (bits & ((1u << len) - 1)))) anyc = 0;
        }
        if (anyc && ye != kReject) {
#pragma unroll
            for (int w = 0; w < WMAX; ++w) ntest += __popc(cm[w]);
            const bword* E = Eall + r * nw * nv;
            bword F[WMAX], FV[WMAX];
#pragma unroll
            for (int w = 0; w < WMAX; ++w) F[w] = FV[w] = 0;
            for (uint32_t y = lo16(ye); y <= hi16(ye); ++y) {
#pragma unroll
                for (int w = 0; w < WMAX; ++w) {
                    if (!EXACTW && static_cast<uint32_t>(w) >= W) continue;
                    F[w] |= E[y * W + w];
                    if (NV) FV[w] |= E[nw + y * W + w];
                }
            }
            const bword* rec = cls + r * cw;
            const uint32_t ncls = rec[0] & 0xFFu;
            if (ncls != 0xFFu) {
                bword U[WMAX], VA[WMAX], OK[WMAX];
#pragma unroll
                for (int w = 0; w < WMAX; ++w) U[w] = VA[w] = OK[w] = 0;
                for (uint32_t c = 0; c < ncls; ++c) {
                    const int ca = hdr_byte(rec, 1 + c);
                    const int cb = hdr_byte(rec, 7 + c);
                    bword win[WMAX], winv[WMAX];
#pragma unroll
                    for (int w = 0; w < WMAX; ++w) win[w] = winv[w] = 0;
                    for (int d = ca; d <= cb; ++d) {
                        or_shifted<WMAX>(F, d, win);
                        if (NV) or_shifted<WMAX>(FV, d, winv);
                    }
#pragma unroll
                    for (int w = 0; w < WMAX; ++w) {
                        if (!EXACTW && static_cast<uint32_t>(w) >= W) continue;
                        const bword m = rec[4 + c * W + w];
                        OK[w] |= m;
                        U[w] |= win[w] & m;
                        if (NV) VA[w] |= winv[w] & m;
                    }
                }
#pragma unroll
                for (int w = 0; w < WMAX; ++w) sw[w] = cm[w] & OK[w] & ~U[w] & (NV ? VA[w] : ~0u);
            } else {
                const uint32_t* xrow = a.xt + (pcol + ja) * n0;
#pragma unroll
                for (int w = 0; w < WMAX; ++w) {
                    bword m = cm[w];
                    while (m) {
                        const uint32_t b = __ffs(m) - 1;
                        m &= m - 1;
                        const uint32_t xe = __ldg(xrow + w * kBits + b);
                        if (xe == kReject) continue;
                        const uint32_t lx = lo16(xe), hx = hi16(xe);
                        bool ok = extract_bits<WMAX>(F, lx, hx) == 0;
                        if (NV) ok = ok && extract_bits<WMAX>(FV, lx, hx) != 0;
                        if (ok) sw[w] |= bword(1) << b;
                    }
                }
            }
        }
#pragma unroll
        for (int w = 0; w < WMAX; ++w)
            if (EXACTW || static_cast<uint32_t>(w) < W) sat[r * nw + i1 * W + w] = sw[w];
    }
    group_sync<WARP>();
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
    if ((tid & 31) == 0 && ntest) atomicAdd(a.stats + kStatsCols * (it + 1) + 2, ntest);
}

// Apply the iteration's hits to word e and build next iteration's D';
// nr / nc collect newly reachable states and newly certified candidates.
// L2: read hit and best[] from L2 (inside the satisfaction kernel, where
// other blocks of the same launch wrote them with atomics and this SM's L1
// may hold an older copy of their lines).
template <bool L2 = false>
__device__ __forceinline__ void finalize_word(const GridInfo& g, const FusedFixArgs& a, const bword* rprev,
                                              bword* rnext, uint64_t e, uint32_t it, unsigned long long& nr,
                                              unsigned long long& nc) {
    const bword rp = rprev[e];
    const bword h = L2 ? __ldcg(a.hit + e) : a.hit[e];
    const bword rn = rp | h;
    rnext[e] = rn;
    const bword dn = (a.validb[e] & ~rn) | a.unsafeb[e];
    if (a.dp[e] & ~dn) {   // the row lost a D' cell in iteration `it`
        const uint32_t r = static_cast<uint32_t>(e / g.W);
        atomicOr(a.rowlost + (it & 1) * a.rl_words + (r >> 5), 1u << (r & 31));
    }
    a.dp[e] = dn;
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
            // Four states at a time: their best[] loads in flight together.
            uint32_t b[4], j[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                b[k] = m ? static_cast<uint32_t>(__ffs(m) - 1) : kBits;
                m &= m - 1;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
                j[k] = b[k] < kBits ? (L2 ? __ldcg(a.best + sbase + b[k]) : a.best[sbase + b[k]]) : kInvalid32;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (b[k] >= kBits) continue;
                const uint64_t s = sbase + b[k];
                a.controller[s] = j[k];
                a.best[s] = kInvalid32;
                if (!((c >> b[k]) & 1u)) a.reach_step[s] = it;
            }
        }
    }
}

// Block-wide: add the block's counters to the iteration's stats row.
__device__ __forceinline__ void add_counters(unsigned long long* row, unsigned long long nr, unsigned long long nc) {
    for (int off = 16; off > 0; off >>= 1) {
        nr += __shfl_down_sync(0xFFFFFFFFu, nr, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nr) atomicAdd(row, nr);
        if (nc) atomicAdd(row + 1, nc);
    }
}

// The stop rules after iteration `it` (reachability.hpp:133-144), by one
// thread once every counter of the iteration is in.
// Its loads are one round, from L2 (where the other blocks' counter atomics
// were performed).
__device__ __forceinline__ void control_step(FixControl* fc, unsigned long long* row, uint32_t it) {
    const unsigned long long tnr = __ldcg(row);
    const unsigned long long tnc = __ldcg(row + 1);
    const unsigned long long certified = __ldcg(&fc->certified) + tnc;
    const unsigned long long reachable = __ldcg(&fc->reachable) + tnr;
    const unsigned long long candidates = __ldcg(&fc->candidate_count);
    const uint32_t max_iterations = __ldcg(&fc->max_iterations);
    const uint32_t stats_cap = __ldcg(&fc->stats_cap);
    fc->certified = certified;
    fc->reachable = reachable;
    fc->iter = it;
    fc->last_new = tnr > 0xFFFFFFFFull ? 0xFFFFFFFFu : static_cast<uint32_t>(tnr);
    if (certified == candidates) {
        fc->converged = 1;
        fc->message = 1;
        fc->stop = 1;
    } else if (tnr == 0 && tnc == 0) {
        fc->message = 2;
        fc->stop = 1;
    } else if (it >= max_iterations || it + 1 >= stats_cap) {
        fc->message = 3;
        fc->stop = 1;
    }
}

}  // namespace fused
}  // namespace gsc_b200
