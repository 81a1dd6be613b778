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

// Word w (0 <= w <= WMAX) of the row F moved by d (|d| < 32): bit j of the
// result is bit 32 w + j + d of F, with F zero outside its WMAX words.
template <int WMAX>
__device__ __forceinline__ bword moved_word(const bword (&F)[WMAX], int w, int d) {
    const bword fm1 = (w >= 1 && w - 1 < WMAX) ? F[w - 1] : 0u;
    const bword f0 = (w < WMAX) ? F[w] : 0u;
    const bword fp1 = (w + 1 < WMAX) ? F[w + 1] : 0u;
    const bool up = d >= 0;
    return __funnelshift_r(up ? f0 : fm1, up ? fp1 : f0, static_cast<uint32_t>(d) & 31u);
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
        // several theta cells are in flight together.  The row-lost words
        // hold W1 = ceil(n1 / 32) words per (theta, v) slice, bit y % 32 of
        // word y / 32 for row y.
        const uint32_t W1 = (n1 + 31) / 32, yw = y >> 5, yb = y & 31;
        uint32_t hit = 0, zz = z;
#pragma unroll 4
        for (uint32_t i = 0; i < kmax; ++i) {
#pragma unroll
            for (uint32_t j = 0; j < kMaxDilate; ++j) {
                if (j < lfit) {
                    hit |= (lost[(zz + n2 * (v + j)) * W1 + yw] >> yb) & 1u;
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
//     the x test 32 states per word: a state whose x box is [i0 + a, i0 + b]
//     is blocked when F has a bit in it, i.e. bit i0 of OR_{d=a..b} (F >> d);
//     with the plane's shift masks M_d (the states whose box holds i0 + d,
//     launch_x_classes) that is bit i0 of OR_d ((F >> d) & M_d), one funnel
//     shift per word and shift for the whole word of states; a plane with
//     boxes of more than kShiftMax shifts is tested state by state;
//  D. per state, the lowest satisfied input of the column goes to best[]
//     (atomicMin, so the lowest over all columns wins) and the hit bit is set.
// WMAX: register words per row; EXACTW: g.W == WMAX (else g.W <= WMAX at run
// time).  NVMODE: 0 / 1 = validity test off / on, 2 = a.need_valid decides.
// WARP: the task is one warp's (its own smem and s_meta), else the block's.
// BULK (one task per block only): phase B stages each representative's rows,
// class record and y table with three 1-D bulk copies (the TMA engine) that
// complete on an mbarrier, instead of one cp.async per word.  A bulk copy
// needs 16-byte aligned ends, so each copies the aligned span around its
// words into a 16-byte aligned slot, and readers add the span's leading
// offset (fused_smem_layout).
// Every early return is taken by the whole group.
// An iteration runs incrementally when the previous one added at most one
// state per kIncrementalRows x-rows.  Measured at 128x128x72x48: 16 -> 4
// took the fixpoint from 42.8 to 40.9 ms; 1 took it to 40.6 ms but slowed
// the published demo by 0.5 %, and testing incrementally in every iteration
// slowed it by 6 %.  A sharded solve sets last_new to 2^32 - 1, which no
// threshold of 1 or more admits.
constexpr unsigned long long kIncrementalRows = 4;

template <int WMAX, bool EXACTW, int NVMODE, bool WARP = false, bool BULK = false>
__device__ __forceinline__ void sat_col_task(const GridInfo& g, const FusedFixArgs& a, uint32_t task,
                                             bword* smem, uint32_t* s_meta) {
    static_assert(!(BULK && WARP), "bulk staging is for one task per block");
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

    const FusedSmemLayout L = fused_smem_layout(nw, nv, mr, cw, n1, ma, BULK);
    bword* act = smem + L.act;
    bword* Eall = smem + L.E;                             // max_reps * nv * L.e_stride
    bword* sat = smem + L.sat;                            // max_reps * nw
    bword* cls = smem + L.cls;                            // max_reps * L.c_stride
    uint32_t* yts = smem + L.yts;                         // max_reps * L.y_stride
    uint32_t* reps = smem + L.reps;                       // ma: acceleration of each representative slot
    uint32_t* repw = reps + ma;                           // ma: its v window
    uint32_t* repo = repw + ma;                           // ma: its part of the dilated rows' offset
    uint32_t* rowchg = smem + L.rowchg;                   // max_reps * W1: y rows of a window that lost a cell
    uint32_t* rsh = smem + L.rsh;                         // BULK, ma: leading offsets of a rep's three spans
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + L.mbar);
    const uint32_t W1 = (n1 + 31) / 32;
    if (BULK && tid == 0) mbar_init(mbar, 1);

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
        // kIncrementalRows x-rows), the iteration runs incrementally (phase
        // B).
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
        if constexpr (BULK) {
            // Warp 0: lane r issues representative r's copies after lane 0
            // has announced every copy's bytes on the barrier.
            if (tid < 32) {
                uint32_t bytes = 0;
                for (uint32_t r = lane; r < nrep; r += 32) {
                    const uint32_t offe = offz + repo[r];
                    const uint64_t pl = pcol + reps[r];
                    const uint32_t she = offe & 3u, shc = static_cast<uint32_t>(pl * cw) & 3u,
                                   shy = static_cast<uint32_t>(pl * n1) & 3u;
                    bytes += 4u * (nv * ((nw + she + 3u) & ~3u) + ((cw + shc + 3u) & ~3u) + ((n1 + shy + 3u) & ~3u));
                }
                for (int off = 16; off > 0; off >>= 1) bytes += __shfl_down_sync(0xFFFFFFFFu, bytes, off);
                if (lane == 0) mbar_arrive_expect_tx(mbar, bytes);
                __syncwarp();
                for (uint32_t r = lane; r < nrep; r += 32) {
                    const uint32_t offe = offz + repo[r];
                    const uint64_t pl = pcol + reps[r];
                    const uint32_t she = offe & 3u;
                    const uint64_t offc = pl * cw, offy = pl * n1;
                    const uint32_t shc = static_cast<uint32_t>(offc) & 3u, shy = static_cast<uint32_t>(offy) & 3u;
                    bword* e0 = Eall + r * nv * L.e_stride;
                    const uint32_t ne = 4u * ((nw + she + 3u) & ~3u);
                    bulk_copy_g2s(e0, a.dzw + (offe - she), ne, mbar);
                    if (NV) bulk_copy_g2s(e0 + L.e_stride, a.vzw + (offe - she), ne, mbar);
                    bulk_copy_g2s(cls + r * L.c_stride, a.xcls + (offc - shc), 4u * ((cw + shc + 3u) & ~3u), mbar);
                    bulk_copy_g2s(yts + r * L.y_stride, a.yt + (offy - shy), 4u * ((n1 + shy + 3u) & ~3u), mbar);
                    rsh[r] = she | (shc << 8) | (shy << 16);
                }
            }
        } else {
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
        }
    };
    if (!incremental) stage();
    int lost = 0;
    if (incremental) {
        const uint32_t* rl = a.rowlost + (it & 1) * a.rl_words;
        for (uint32_t e = tid; e < nrep * W1; e += bd) {
            const uint32_t r = e / W1, yw = e - r * W1;
            const uint32_t we = repw[r];
            const uint32_t v0 = lo16(we), v1 = hi16(we);
            // The window's (theta, v) slices' row-lost words (W1 per slice),
            // the next slice's load issued before the current one is used.
            uint32_t z = lz, v = v0;
            uint32_t c0 = __ldg(rl + (z + n2 * v) * W1 + yw);
            uint32_t m = 0;
            for (uint32_t q = 1; q < nz * (v1 - v0 + 1); ++q) {
                if (v == v1) {
                    v = v0;
                    z = (z + 1 == n2) ? 0 : z + 1;
                } else {
                    ++v;
                }
                const uint32_t d0 = __ldg(rl + (z + n2 * v) * W1 + yw);
                m |= c0;
                c0 = d0;
            }
            m |= c0;
            rowchg[r * W1 + yw] = m;
            lost |= m != 0;
        }
    }
    if (incremental) {
        if (!group_sync_or<WARP>(lost)) return;
        stage();
    }
    if constexpr (BULK) {
        // Bounded wait for the copies.  A wait that gives up (it cannot in a
        // working device: the copies are a few KB) stops the solve with
        // kMsgDeviceTimeout, which the host reports as GSC_ERR_TIMEOUT, and
        // waits once more, again bounded, before the block leaves.
        bool done = false;
        for (uint32_t k = 0; k < kBulkWaitProbes && !done; ++k) done = mbar_try_wait(mbar, 0);
        if (!done) {
            FixControl* wfc = a.fc;
            wfc->message = kMsgDeviceTimeout;
            atomicExch(&wfc->stop, 1u);
            for (uint32_t k = 0; k < kBulkWaitProbes && !done; ++k) done = mbar_try_wait(mbar, 0);
        }
        if (group_sync_or<WARP>(done ? 0 : 1)) return;
    } else {
        cp_async_wait_all();
        group_sync<WARP>();
    }
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
        const uint32_t rs = BULK ? rsh[r] : 0u;
        const uint32_t ye = BULK ? yts[r * L.y_stride + (rs >> 16) + i1] : yts[r * n1 + i1];
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
            const bword* E = BULK ? Eall + r * nv * L.e_stride + (rs & 0xFFu) : Eall + r * nw * nv;
            const uint32_t ev = BULK ? L.e_stride : nw;   // the valid rows follow the D' rows
            bword F[WMAX], FV[WMAX];
#pragma unroll
            for (int w = 0; w < WMAX; ++w) F[w] = FV[w] = 0;
            for (uint32_t y = lo16(ye); y <= hi16(ye); ++y) {
#pragma unroll
                for (int w = 0; w < WMAX; ++w) {
                    if (!EXACTW && static_cast<uint32_t>(w) >= W) continue;
                    F[w] |= E[y * W + w];
                    if (NV) FV[w] |= E[ev + y * W + w];
                }
            }
            const bword* rec = BULK ? cls + r * L.c_stride + ((rs >> 8) & 0xFFu) : cls + r * cw;
            const bword hdr = rec[0];
            const uint32_t nd = hdr & 0xFFu;
            if (nd != 0xFFu) {
                // U = OR_d ((F >> d) & M_d) over the plane's shifts (and VA
                // likewise over the valid rows): G is F moved by dmin, one
                // word longer, so every shift is a right funnel shift by
                // d - dmin in [0, kShiftMax).
                const int dmin = static_cast<int8_t>((hdr >> 8) & 0xFFu);
                bword G[WMAX + 1], GV[WMAX + 1];
#pragma unroll
                for (int w = 0; w <= WMAX; ++w) {
                    G[w] = moved_word<WMAX>(F, w, dmin);
                    GV[w] = NV ? moved_word<WMAX>(FV, w, dmin) : 0u;
                }
                bword U[WMAX], VA[WMAX];
#pragma unroll
                for (int w = 0; w < WMAX; ++w) U[w] = VA[w] = 0;
                for (uint32_t i = 0; i < nd; ++i) {
#pragma unroll
                    for (int w = 0; w < WMAX; ++w) {
                        if (!EXACTW && static_cast<uint32_t>(w) >= W) continue;
                        const bword m = rec[4 + i * W + w];
                        U[w] |= __funnelshift_r(G[w], G[w + 1], i) & m;
                        if (NV) VA[w] |= __funnelshift_r(GV[w], GV[w + 1], i) & m;
                    }
                }
#pragma unroll
                for (int w = 0; w < WMAX; ++w) {
                    const bword ok = (EXACTW || static_cast<uint32_t>(w) < W) ? rec[4 + kShiftMax * W + w] : 0u;
                    sw[w] = cm[w] & ok & ~U[w] & (NV ? VA[w] : ~0u);
                }
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
// The reachable set is updated in place (rprev and rnext name one buffer),
// and D' = (valid & ~reachable) | unsafe holds for every word between
// iterations, so a word without a hit keeps all of its bits: its thread
// reads the hit word and stops.
__device__ __forceinline__ void finalize_word(const GridInfo& g, const FusedFixArgs& a, const bword* rprev,
                                              bword* rnext, uint64_t e, uint32_t it, unsigned long long& nr,
                                              unsigned long long& nc) {
    const bword h = a.hit[e];
    if (!h) return;
    // Every load the word needs, issued before any of its stores (one round
    // trip): its sets and the best[] entries of its first four new states.
    const bword rp = rprev[e];
    const bword vb = a.validb[e], ub = a.unsafeb[e], dpo = a.dp[e], c = a.candb[e], act = a.active[e];
    const uint64_t r = e / g.W;
    const uint64_t sbase = r * g.n[0] + (e - r * g.W) * kBits;
    bword m = h;
    uint32_t b[4], j[4];
    // Four states at a time: their best[] loads in flight together.
    auto load4 = [&]() {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            b[k] = m ? static_cast<uint32_t>(__ffs(m) - 1) : kBits;
            m &= m - 1;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) j[k] = b[k] < kBits ? a.best[sbase + b[k]] : kInvalid32;
    };
    load4();
    const bword rn = rp | h;
    rnext[e] = rn;
    const bword dn = (vb & ~rn) | ub;
    if (dpo & ~dn) {   // the row lost a D' cell in iteration `it`: word y / 32 of its slice
        const uint32_t row = static_cast<uint32_t>(r), n1 = g.n[1];
        const uint32_t sl = row / n1, y = row - sl * n1;
        atomicOr(a.rowlost + (it & 1) * a.rl_words + sl * ((n1 + 31) / 32) + (y >> 5), 1u << (y & 31));
    }
    a.dp[e] = dn;
    a.hit[e] = 0;
    a.active[e] = act & ~h;
    nr += __popc(h & ~rp);
    nc += __popc(h & c);
    for (;;) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (b[k] >= kBits) continue;
            const uint64_t s = sbase + b[k];
            a.controller[s] = j[k];
            a.best[s] = kInvalid32;
            if (!((c >> b[k]) & 1u)) a.reach_step[s] = it;
        }
        if (!m) break;
        load4();
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

// iter | stop << 32 of the control record into the host's mirror word, for
// a host loop that polls it instead of copying the record back.
__device__ __forceinline__ void write_mirror(unsigned long long* mirror, const FixControl* fc) {
    *reinterpret_cast<volatile unsigned long long*>(mirror) =
        fc->iter | (static_cast<unsigned long long>(fc->stop ? 1u : 0u) << 32);
    __threadfence_system();
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
