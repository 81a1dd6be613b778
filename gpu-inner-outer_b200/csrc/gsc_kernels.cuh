// gsc_kernels.cuh -- launch wrappers shared between the kernel files and the C ABI layer.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gsc_common.cuh"

namespace gsc_b200 {

// Launch of `k` that may begin while the kernel queued before it on `st`
// drains (programmatic stream serialization); `k` starts with pdl_wait().
// Under stream capture the dependency becomes a programmatic graph edge.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

// ---- abstraction (resident nominal successors) ------------------------------------------
// xn[((i2*n3 + i3)*M + j)*n0 + i0] = nominal x after K Euler substeps (model.hpp:26-46),
// yn likewise over i1.  cosT/sinT[(i2*mw + jw)*K + k], vseq[(i3*ma + ja)*K + k].
cudaError_t launch_nominal_xy(const GridInfo& g, const double* cosT, const double* sinT, const double* vseq,
                              double* xn, double* yn, cudaStream_t st);

// ---- query preparation ------------------------------------------------------------------
struct MaskArgs {
    const double* obstacles;  // [n][8] device
    uint8_t* valid;           // [S]
    uint8_t* cand;            // [S]
    int build_valid;          // 0: valid already filled by the caller's mask
    int build_cand;
    const uint8_t* safe;      // caller's constraint mask (rank 2 or 4), or null: use the constraint kind
    int safe_rank;
    const uint8_t* cmp_safe;  // safety at the centres (rank cmp_rank), to count cells whose validity differs
    int cmp_rank;
    unsigned long long* counts;  // [0] valid, [1] candidate, [2] candidate-not-valid, [4] valid != safe
};
cudaError_t launch_masks(const GridInfo& g, const QueryInfo& q, const MaskArgs& a, cudaStream_t st);
cudaError_t launch_safe2(const GridInfo& g, const QueryInfo& q, uint8_t* safe2, cudaStream_t st);

// Per-axis quantised boxes.  xt/yt: [n2][n3][M][n0|n1], zt: [n2][mw], wt: [n3][ma], packed
// lo | hi << 16 or kReject.  flags |= 1 if an accepted non-wrap interval is empty (hi < lo),
// |= 2 if one is wider than 64 cells.
cudaError_t launch_axis_tables(const GridInfo& g, const QueryInfo& q, const double* xn, const double* yn,
                               const double* thf, const double* vf, uint32_t* xt, uint32_t* yt, uint32_t* zt,
                               uint32_t* wt, unsigned int* flags, cudaStream_t st);

// Bit-sliced sets: bit b of word w of x-row r is state r*n0 + 32*w + b.
// mode 0: bit = src[s] != 0; 1: bit = src[s] == 0; 2: bit = src2d[i1*n0 + i0] == 0;
// 3: bit = src[s] != 0 && src2d[i1*n0+i0] != 0; 4: bit = src[s] != 0 && src[s] (4-D second) != 0
cudaError_t launch_pack_bits(const GridInfo& g, int mode, const uint8_t* src, const uint8_t* src2, bword* out,
                             cudaStream_t st);
cudaError_t launch_unpack_bits(const GridInfo& g, const bword* bits, uint8_t* out, cudaStream_t st);
// n words from src to dst by one small kernel (dst may be pinned host memory
// mapped into the device's address space).
cudaError_t launch_store_words(const uint32_t* src, uint32_t* dst, uint32_t n, cudaStream_t st);
// The fixpoint's current reachable set (reach0 or reach1 by fc->iter, read
// on the device) as one byte per state.
cudaError_t launch_unpack_reach(const GridInfo& g, const FixControl* fc, const bword* reach0, const bword* reach1,
                                uint8_t* out, cudaStream_t st);

// ---- 4-D inclusive prefix tables (int32, zero first plane per dimension) -----------------
// mode 0: valid; 1: valid && !reach (b = reach); 2: !safe (4-D safe mask).
// Built in two passes (x-y per (theta, v) slice, then theta-v per (x tile,
// y)) when a slice and a theta-v plane fit shared memory, else one pass per
// dimension.  ev (optional, prefix4_launches(g) events): ev[k] is recorded
// after pass k + 1.
cudaError_t launch_prefix4(const GridInfo& g, int mode, const uint8_t* a, const uint8_t* b, int32_t* table,
                           const FixControl* ctl, cudaStream_t st, cudaEvent_t* ev = nullptr);
// Kernels launch_prefix4 launches for this grid.
uint32_t prefix4_launches(const GridInfo& g);
// 2-D prefix of !safe2 over (x, y): (n0+1)*(n1+1) entries, stride n0+1.
cudaError_t launch_prefix2_unsafe(const GridInfo& g, const uint8_t* safe2, int32_t* table, cudaStream_t st);

// ---- stored per-pair boxes --------------------------------------------------------------
struct StoredBuildArgs {
    const uint32_t *xt, *yt, *zt, *wt;
    const uint8_t* safe;      // rank 2 or 4
    int safe_rank;
    const int32_t* unsafe2;   // rank 2 prefix
    const int32_t* unsafe4;   // rank 4 prefix
    const int32_t* pvalid;    // 4-D valid prefix
    uint2* boxes;             // [M][S_pad]: one byte per bound (every dimension <= 255 cells)
    uint64_t S_pad;
    uint4* boxes16;           // [M][S]: 16 bits per bound, when a dimension has more than 255 cells
    int wide;                 // 1: boxes16 in use
    unsigned long long* valid_pairs;   // abstraction-valid pairs (before the V(box) > 0 fold)
};
cudaError_t launch_stored_build(const GridInfo& g, const StoredBuildArgs& a, cudaStream_t st);

// Reference-format abstraction (pair = s * M + j), abstraction.hpp:161-209.
struct ExportArgs {
    const uint32_t *xt, *yt, *zt, *wt;
    const uint8_t* safe;
    int safe_rank;
    const int32_t* unsafe2;
    const int32_t* unsafe4;
    uint32_t* min_flat;
    uint32_t* max_flat;
    uint8_t* valid;
    uint64_t pair_begin, pair_count;
};
cudaError_t launch_export(const GridInfo& g, const ExportArgs& a, cudaStream_t st);

// ---- fixpoint ---------------------------------------------------------------------------
struct StoredFixArgs {
    const uint2* boxes;
    uint64_t S_pad;
    const uint4* boxes16;     // wide grids: {lo0 | lo1 << 16, lo2 | lo3 << 16, hi0 | hi1 << 16, hi2 | hi3 << 16}
    int wide;
    int32_t* pd;              // D-prefix table
    const uint8_t* valid;
    const uint8_t* cand;
    uint8_t* reach;
    uint32_t* controller;
    uint32_t* reach_step;
    FixControl* fc;
    unsigned long long* stats;   // [stats_cap][kStatsCols]
    cudaGraphConditionalHandle cond;
    int use_cond;
    // Host-loop solves: a word of page-locked host memory, mapped for the
    // device, that receives iter | stop << 32 after each iteration's stop
    // rules (write_mirror), or nullptr.
    unsigned long long* mirror;
};
cudaError_t launch_stored_init(const GridInfo& g, const StoredFixArgs& a, cudaStream_t st);
// ev (optional, kProfileEvents events): [0] before the prefix rebuild,
// [1..n] after its n passes (launch_prefix4: n = prefix4_launches(g); events
// n+1 .. 4 are not recorded), [5] after the satisfaction kernel, [6] after
// the control kernel.  The fused iteration records [0], [1] after the
// dilation, [5] and [6] alike.
constexpr int kProfileEvents = 8;
cudaError_t launch_stored_iteration(const GridInfo& g, const StoredFixArgs& a, cudaStream_t st, uint32_t* launches,
                                    cudaEvent_t* ev = nullptr);
// One thread that holds the stream for about `ns` nanoseconds (bounded by
// the global timer and by an iteration cap), so that what the host queues
// behind it meanwhile runs back to back: profiled phases then time the
// kernels rather than the host's enqueueing.
cudaError_t launch_hold(cudaStream_t st, uint64_t ns);

// Box widths present in a problem: theta widths kval[0..nk) and v widths
// lval[0..nl), ascending; combo (ki, li) indexes the dilated copies.
constexpr int kMaxDilate = 8;
struct DilateArgs {
    uint32_t nk, nl;
    uint32_t kval[kMaxDilate];
    uint32_t lval[kMaxDilate];
};

// Set-up plan of a problem, written by k_plan and copied to the host once:
// the mask counts and axis-table flags, the largest number of representative
// accelerations in one omega column, and the theta / v box widths in use.
struct PlanRecord {
    unsigned long long counts[8];
    uint32_t flags;
    uint32_t max_reps;
    uint32_t width_overflow;   // more widths than kMaxDilate, or a v width above kMaxDilate
    uint32_t fused;            // 1 when the fused tables were planned
    DilateArgs dil;
};

struct FusedFixArgs {
    const uint32_t *xt, *yt, *zt, *wt;
    const bword* validb;
    const bword* unsafeb;
    const bword* srcb;         // valid && source-safe
    const bword* candb;
    bword* dp;
    bword* reach0;
    bword* reach1;             // the same buffer as reach0: the reachable set is updated in place
    bword* active;
    bword* hit;                // states satisfied this iteration (cleared by the finalize kernel)
    uint32_t* best;            // lowest satisfied input per state this iteration (else 0xFFFFFFFF)
    uint32_t* controller;
    uint32_t* reach_step;
    FixControl* fc;
    unsigned long long* stats;
    int need_valid;
    const bword* xcls;         // per-plane x-box classes (launch_x_classes)
    const uint8_t* xrep;       // per plane: the first acceleration of its omega column with identical boxes
    uint32_t cls_words;        // 32-bit words per class record
    uint32_t max_reps;         // max representative accelerations of one omega column
    uint32_t sat_threads;      // threads per satisfaction block (64, 128 or 256)
    bword* dzw;                // (theta, v)-dilated D' [combo][rows * W], brought up to date each iteration
    uint32_t* rowlost;         // [2][rl_words] bit per x-row: the row lost a D' cell in the iteration
                               // (W1 = ceil(n1 / 32) words per (theta, v) slice, bit y % 32 of word y / 32)
                               // (iter & 1) just finalised
    uint32_t rl_words;         // rows / 32 + 2
    const bword* vzw;          // (theta, v)-dilated valid set (when validity is more than safety)
    const uint8_t* kidx;       // [n2 + 1]: theta width -> its slot in dil.kval
    const uint8_t* lidx;       // [n3 + 1]: v width -> its slot in dil.lval
    uint32_t nl;
    DilateArgs dil;
    // Word offset of a representative's dilated D' row 0 in dzw, split into
    // a part per omega column and theta cell and a part per acceleration and
    // v cell (sums modulo 2^32, as dzw offsets are 32-bit):
    const uint32_t* offz;      // [n2 * mw]: kslot * nl * rows * W + n1 * lz * W
    const uint32_t* offv;      // [n3 * ma]: lslot * rows * W + n1 * n2 * lw * W
    // Sharded solve (one rank of several): the satisfaction launch covers
    // slices [shard_begin, shard_begin + shard_slices) only, and the stop
    // rules are left to the host, which applies them with the counts of
    // every rank (gsc_problem_shard_control).  shard_slices == 0: not sharded.
    uint32_t shard_begin;
    uint32_t shard_slices;
    cudaGraphConditionalHandle cond;
    int use_cond;
    unsigned long long* mirror;   // as StoredFixArgs::mirror
};
constexpr int kFusedWarps = 8;   // most warps of a satisfaction block

// Shared-memory layout of one satisfaction task, in 32-bit words: the
// active rows, the representatives' dilated D' (and valid) rows, their
// satisfied masks, class records and y tables, the representatives' index,
// v window and offset part, the changed-row masks, and with bulk staging
// the spans' leading offsets and the mbarrier.  Bulk staging gives every
// staged span a 16-byte aligned slot three words longer than its data.
struct FusedSmemLayout {
    uint32_t act, E, sat, cls, yts, reps, rowchg, rsh, mbar, total;
    uint32_t e_stride, c_stride, y_stride;
};
__host__ __device__ inline FusedSmemLayout fused_smem_layout(uint32_t nw, uint32_t nv, uint32_t mr, uint32_t cw,
                                                             uint32_t n1, uint32_t ma, bool bulk) {
    auto r4 = [](uint32_t x) { return (x + 3u) & ~3u; };
    const uint32_t w1 = (n1 + 31) / 32;
    FusedSmemLayout L;
    L.act = 0;
    L.e_stride = bulk ? r4(nw + 3) : nw;
    L.c_stride = bulk ? r4(cw + 3) : cw;
    L.y_stride = bulk ? r4(n1 + 3) : n1;
    L.E = bulk ? r4(nw) : nw;
    L.sat = L.E + mr * nv * L.e_stride;
    L.cls = bulk ? r4(L.sat + mr * nw) : L.sat + mr * nw;
    L.yts = L.cls + mr * L.c_stride;
    L.reps = L.yts + mr * L.y_stride;
    L.rowchg = L.reps + 3 * ma;
    L.rsh = L.rowchg + mr * w1;
    L.mbar = bulk ? ((L.rsh + ma + 1) & ~1u) : L.rsh;
    L.total = bulk ? L.mbar + 2 : L.rsh;
    return L;
}
constexpr int kShiftMax = 8;   // most shifts d of a plane's shift-mask record
constexpr size_t kFusedSmemMax = 200 * 1024;
// Dynamic shared memory of one fused satisfaction task (bulk: the
// one-problem kernel's bulk-staged layout; else the batched kernels').
size_t fused_smem_bytes(const GridInfo& g, uint32_t cls_words, int need_valid, uint32_t max_reps, bool bulk);
// Threads per satisfaction block for a problem: 128, or 256 when a block has
// more representative rows to stage and test (max_reps * n1 * W words above
// 2304).  128 measured 1 % faster than 64 at 65x65x38x25 and equal on the
// published demo.
uint32_t fused_sat_threads(const GridInfo& g, uint32_t max_reps);
// Dilated copies of src into dst.  With fc and rowlost (during a fixpoint,
// after its first iteration) only positions whose window holds a row that
// lost a D' cell are recomputed; it also clears the row bits the next
// finalize writes.
cudaError_t launch_dilate(const GridInfo& g, const bword* src, bword* dst, const DilateArgs& d, const FixControl* fc,
                          uint32_t* rowlost, uint32_t rl_words, cudaStream_t st);
// Fills a PlanRecord from the counts, flags and (when xrep is set) the
// theta / v tables and plane representatives; writes kidx / lidx.
cudaError_t launch_plan(const GridInfo& g, const uint32_t* zt, const uint32_t* wt, const uint8_t* xrep,
                        const unsigned long long* counts, const unsigned int* flags, uint8_t* kidx, uint8_t* lidx,
                        PlanRecord* out, cudaStream_t st);
// One instance of a batched solve (or of the serving loop), resident in
// device memory and indexed by slot.
struct InstanceDesc {
    GridInfo g;
    FusedFixArgs a;
    const uint8_t* cand;
    const unsigned long long* counts;
    uint32_t max_iterations;
    uint32_t stats_cap;
    uint32_t sat_tasks;   // slices * mw
    uint32_t words;       // rows * W
};

// The instances one launch works on: slot[k] and, per task kind, the prefix
// offsets of their tasks (off[0] = 0, off[n] = total).  A dilate / finalize
// task covers `chunk` word positions; an init task `chunk` words, states and
// stats entries.
struct WorkList {
    const uint32_t* slot;
    const uint32_t* sat_off;
    const uint32_t* dil_off;
    const uint32_t* fin_off;
    const uint32_t* ini_off;
    uint32_t n;
    uint32_t chunk;
    FixControl* status;   // [n]: copy of each instance's FixControl after the iteration (optional)
    uint32_t* running;    // instances still running after the iteration (optional)
};

// Launch shapes of the batched kernels.
struct BatchShape {
    uint32_t sat_threads;   // threads per satisfaction block
    uint32_t sat_blocks;    // persistent satisfaction blocks (0 = one per task)
    uint32_t chunk;         // word positions per dilate / finalize task
    uint32_t warp;          // 1: one satisfaction task per warp (smem per task, sat_threads / 32 of them)
};

// Host-side task counts of one list (matching WorkList's offsets).
struct WorkTotals {
    uint32_t sat, dil, fin, ini;
};

// An instance of a batch that keeps the GPU busy on its own (at least
// kBigPairs state-input pairs per iteration) iterates with the one-problem
// kernels, whose row width is a compile-time constant and whose arguments
// stay in the constant bank.  Smaller instances gain more from sharing the
// batched kernels' launches than they lose to their run-time row width.
constexpr uint64_t kBigPairs = 1ull << 28;
inline bool is_big_instance(const GridInfo& g) { return g.S * g.M >= kBigPairs; }

// A big instance of a batch: its grid and its fixpoint arguments (without a
// graph condition; the batch's status kernel sets that).
struct BigInstance {
    GridInfo g;
    FusedFixArgs a;
};

cudaError_t launch_batch_init(const InstanceDesc* descs, const WorkList& wl, const WorkTotals& tot, int sms,
                              cudaStream_t st);
// One fixpoint iteration of every listed instance: dilate, satisfaction,
// finalize and status (which also sets the graph condition when use_cond).
cudaError_t launch_batch_iteration(const InstanceDesc* descs, const WorkList& wl, const WorkTotals& tot,
                                   const BatchShape& sh, uint32_t wmax, size_t smem, int sms,
                                   cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st,
                                   uint32_t* launches);
// One fixpoint iteration of a mixed batch: each of the nbig big instances
// with the one-problem kernels, the instances of `small` with the batched
// kernels (wmax and smem are theirs), then the status kernel over `all`
// (every instance, big and small, in the order its status records use).
cudaError_t launch_batch_step(const InstanceDesc* descs, const WorkList& small, const WorkTotals& tot_small,
                              const WorkList& all, const BigInstance* big, uint32_t nbig, const BatchShape& sh,
                              uint32_t wmax, size_t smem, int sms, cudaGraphConditionalHandle cond, int use_cond,
                              cudaStream_t st, uint32_t* launches);
// Dynamic shared memory of one satisfaction block for a shape, given one
// task's staging (smem).
inline size_t batch_sat_smem(const BatchShape& sh, size_t smem) { return sh.warp ? (sh.sat_threads / 32) * smem : smem; }

// Shift-mask record words per plane: a 16-byte header + (kShiftMax + 1) * W masks.
__host__ __device__ inline uint32_t class_words(const GridInfo& g) { return 4 + (kShiftMax + 1) * g.W; }
// Per (slice, input) plane, the x boxes [i0 + a, i0 + b] of its states as
// shift masks: M_d = the states whose box holds i0 + d, for the nd shifts
// d = dmin .. dmin + nd - 1 (nd <= kShiftMax), and OK = the states with a
// box.  A state is blocked by a row F exactly when bit i0 of
// OR_d ((F >> d) & M_d) is set.  Header word 0: byte 0 = nd (0xFF: the plane
// is irregular and tested state by state), byte 1 = dmin (int8); then M_d
// for each d (W words each) at word 4 + (d - dmin) * W, and OK at word
// 4 + kShiftMax * W.  |a|, |b| < 32.
cudaError_t launch_x_classes(const GridInfo& g, const uint32_t* xt, bword* xcls, cudaStream_t st);
// Per plane (slice, j = ja + ma * jw): the lowest ja' of the same omega column
// whose x row, y row and v box equal those of ja, so the two inputs test every
// state alike (with one Euler substep the x and y successors do not depend on
// the acceleration at all).
// Also raises *max_reps to the most representatives of one omega column.
cudaError_t launch_plane_reps(const GridInfo& g, const uint32_t* xt, const uint32_t* yt, const uint32_t* wt,
                              uint8_t* xrep, uint32_t* max_reps, cudaStream_t st);
cudaError_t launch_fused_init(const GridInfo& g, const FusedFixArgs& a, const uint8_t* cand, cudaStream_t st);
// The offz / offv tables of a problem (after its plan: kidx, lidx, nl).
cudaError_t launch_sat_offsets(const GridInfo& g, const uint32_t* zt, const uint32_t* wt, const uint8_t* kidx,
                               const uint8_t* lidx, uint32_t nl, uint32_t* offz, uint32_t* offv, cudaStream_t st);
// One iteration is three launches: the dilation, the satisfaction kernel
// and the finalize kernel (whose last block applies the stop rules).
// ev (optional, kProfileEvents events): [0] before the dilation, [1..4] after
// it, [5] after the satisfaction kernel, [6] after the finalize kernel.
cudaError_t launch_fused_iteration(const GridInfo& g, const FusedFixArgs& a, cudaStream_t st, uint32_t* launches,
                                   cudaEvent_t* ev = nullptr);

// Sharded solve: the iteration's dilation (of the whole grid) and
// satisfaction (of the shard's slices) without the stop rules.
cudaError_t launch_shard_iteration(const GridInfo& g, const FusedFixArgs& a, cudaStream_t st);
// Stop rules of a sharded solve's iteration fc->iter + 1 with the counts of
// every rank; the next iteration is never incremental.
cudaError_t launch_shard_control(FixControl* fc, unsigned long long* stats, unsigned long long new_reachable,
                                 unsigned long long new_certified, cudaStream_t st);

// Resets the control block and zeroes the per-iteration counters.
cudaError_t launch_fix_init(FixControl* fc, uint32_t max_iterations, uint32_t stats_cap,
                            const unsigned long long* counts, unsigned long long* stats, cudaStream_t st);

// Sets the graph condition from the control block (first node of a graph solve).
cudaError_t launch_set_condition(const FixControl* fc, cudaGraphConditionalHandle cond, cudaStream_t st);

}  // namespace gsc_b200
