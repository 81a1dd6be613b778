// gsc_common.cuh -- shared device/host definitions of the B200 grid symbolic-control library.
//
// Notation: S states (cells), M inputs, P = S * M pairs.  States are x-fastest
// (grid.hpp:126-129): s = i0 + n0 * (i1 + n1 * (i2 + n2 * i3)), dimension 2
// (theta) wraps.  Inputs are j = ja + ma * jw with ja on input dim 0 (the
// acceleration a) and jw on input dim 1 (the turn rate omega) (grid.hpp:68-78).
//
// Exactness: every double operation on the successor-box path uses an
// explicitly rounded intrinsic (__dmul_rn, __dadd_rn, __dsub_rn, __ddiv_rn),
// which nvcc never contracts into FMA, in the reference's operation order
// (model.hpp:26-112, grid.hpp:38-44, grid.hpp:181-251).  cos/sin are never
// evaluated on the device: the host tabulates them with the C library that the
// reference itself calls (model.hpp:36-37).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gsc_b200 {

constexpr uint32_t kInvalid32 = 0xFFFFFFFFu;   // kInvalidInput / kUnreachableStep (types.hpp:22-23)
constexpr uint32_t kReject = 0xFFFFFFFFu;      // axis-table entry of a bounds-rejected pair
constexpr uint32_t kBoxSentinel = 0xFFFFFFFFu; // stored-box entry of an invalid pair
// Bit-sliced sets use 32-bit words: every shift of a row is one native
// funnel shift.  A row of n0 x-cells takes W = ceil(n0 / 32) words.
using bword = uint32_t;
constexpr int kBits = 32;
constexpr int kMaxWords = 8;                   // bit-sliced rows: n0 <= 256
// Per-iteration counters: [0] newly reachable, [1] newly certified candidates,
// [2] pair tests performed (stored: boxes streamed; fused: (state, input)
// tests), [3] stored: box counts evaluated; fused: (slice, input) plane tasks.
constexpr int kStatsCols = 4;

// Geometry shared by all kernels (by value in kernel parameters).
struct GridInfo {
    double lb[4], ub[4], eta[4];
    uint32_t n[4];
    double ilb[2], ieta[2];
    uint32_t ma, mw, M;
    double T;
    uint32_t K;          // integration substeps
    double dt;           // T / K (model.hpp:33)
    uint64_t S;          // states
    uint32_t ps[4];      // padded prefix strides (grid.hpp:253-269)
    uint64_t tsize;      // padded prefix entries
    uint32_t W;          // 32-bit words per x-row of a bit-sliced set
    uint64_t rows;       // n1 * n2 * n3 x-rows
    uint32_t slices;     // n2 * n3 (theta, v) slices
    uint32_t magic_n1;   // fdiv(x, n1) / fdiv(x, n1 * W) multipliers (see fdiv)
    uint32_t magic_nw;
};

// x / d for x * d < 2^32 with m = floor(2^32 / d) + 1 (m = 0 encodes d = 1).
__host__ __device__ __forceinline__ uint32_t fdiv_magic(uint32_t d) {
    return d <= 1 ? 0u : static_cast<uint32_t>((1ull << 32) / d + 1);
}
__device__ __forceinline__ uint32_t fdiv(uint32_t x, uint32_t m) { return m ? __umulhi(x, m) : x; }

// Programmatic dependent launch (PTX griddepcontrol, sm_90 and later): wait
// until the kernel this one was launched after has completed and its writes
// are visible.  Called first in a kernel, before any load or store of global
// memory.  The launch of such a kernel is prepared while its predecessor
// runs and its blocks start as the predecessor's blocks exit (no explicit
// early trigger: releasing dependents at the start of a kernel measured
// slower).  For a kernel launched without the programmatic-serialization
// attribute the instruction has no effect.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Per-query constants.
struct QueryInfo {
    double dhw[4];
    int32_t ckind;
    double cp[4];
    double map_lb[4], map_ub[4];
    int32_t n_obstacles;
    int32_t cand_kind;
    double cand[8];
    uint32_t max_iterations;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Cell centre along one dimension: lb + (i + 0.5) * eta (grid.hpp:38-44).
__device__ __forceinline__ double centre(const GridInfo& g, int d, uint32_t i) {
    return dadd(g.lb[d], dmul(dadd(static_cast<double>(i), 0.5), g.eta[d]));
}

// Input centre along one input dimension (grid.hpp:68-78).
__device__ __forceinline__ double input_centre(const GridInfo& g, int d, uint32_t i) {
    return dadd(g.ilb[d], dmul(dadd(static_cast<double>(i), 0.5), g.ieta[d]));
}

// Successor-box radius along dimension d for a source speed centre v
// (model.hpp:55-76 and :84-89, summed as in :107-111).
__device__ __forceinline__ double box_radius(const GridInfo& g, const QueryInfo& q, int d, double v) {
    const double he0 = dmul(0.5, g.eta[0]);
    const double he1 = dmul(0.5, g.eta[1]);
    const double he2 = dmul(0.5, g.eta[2]);
    const double he3 = dmul(0.5, g.eta[3]);
    const double T = g.T;
    double jfx;
    if (d == 0 || d == 1) {
        const double abs_v = fabs(v);
        jfx = dadd(dadd(d == 0 ? he0 : he1, dmul(dmul(T, abs_v), he2)), dmul(T, he3));
    } else {
        jfx = (d == 2) ? he2 : he3;
    }
    return dadd(jfx, dmul(T, q.dhw[d]));
}

// Quantise [lo_c, hi_c] to clamped cell indices (grid.hpp:222-247).
__device__ __forceinline__ void quantise(const GridInfo& g, int d, double lo_c, double hi_c, uint32_t* lo,
                                         uint32_t* hi) {
    long long lower = static_cast<long long>(floor(ddiv(dsub(lo_c, g.lb[d]), g.eta[d])));
    long long upper = static_cast<long long>(ceil(ddiv(dsub(hi_c, g.lb[d]), g.eta[d]))) - 1;
    const long long n = static_cast<long long>(g.n[d]);
    if (lower < 0) lower = 0;
    if (upper < 0) upper = 0;
    if (lower >= n) lower = n - 1;
    if (upper >= n) upper = n - 1;
    *lo = static_cast<uint32_t>(lower);
    *hi = static_cast<uint32_t>(upper);
}

// Non-wrap dimension: bounds rejection with 1e-9 slack (grid.hpp:187-194),
// then quantisation.  Returns false when rejected.
__device__ __forceinline__ bool axis_box(const GridInfo& g, int d, double nominal, double radius, uint32_t* lo,
                                         uint32_t* hi) {
    const double kEps = 1e-9;
    const double mn = dsub(nominal, radius);
    const double mx = dadd(nominal, radius);
    if (mn < dsub(g.lb[d], kEps) || mx > dadd(g.ub[d], kEps)) return false;
    quantise(g, d, mn, mx, lo, hi);
    return true;
}

// grid.hpp:46-57.
__device__ __forceinline__ double wrap_value(const GridInfo& g, double x) {
    const double low = g.lb[2];
    const double high = g.ub[2];
    const double span = dsub(high, low);
    while (x < low) x = dadd(x, span);
    while (x >= high) x = dsub(x, span);
    return x;
}

// Wrapped dimension 2 (grid.hpp:196-220): full circle when the box is at
// least one span wide, otherwise both ends wrapped then quantised; lo > hi
// marks a box that crosses the seam.
__device__ __forceinline__ void wrap_box(const GridInfo& g, double nominal, double radius, uint32_t* lo,
                                         uint32_t* hi) {
    const double kEps = 1e-9;
    const double mn = dsub(nominal, radius);
    const double mx = dadd(nominal, radius);
    const double wrap_span = dsub(g.ub[2], g.lb[2]);
    const double raw = dsub(mx, mn);
    if (raw >= dsub(wrap_span, kEps)) {
        *lo = 0;
        *hi = g.n[2] - 1;
        return;
    }
    quantise(g, 2, wrap_value(g, mn), wrap_value(g, mx), lo, hi);
}

// config.cpp:62-75 and the quadric predicate; x = cell centre.
__device__ __forceinline__ bool satisfies(const QueryInfo& q, double x0, double x1) {
    switch (q.ckind) {
        case 0:
            return true;
        case 1: {
            const double x1_sq = dmul(x0, x0);
            const double x2_sq = dmul(x1, x1);
            return (dsub(x1_sq, x2_sq) <= q.cp[0]) && (dsub(dmul(q.cp[1], x2_sq), x1_sq) <= q.cp[2]);
        }
        case 2: {
            const double a = ddiv(x0, q.cp[0]);
            const double b = ddiv(x1, q.cp[1]);
            return dadd(dmul(a, a), dmul(b, b)) <= 1.0;
        }
        case 3:
            return (dsub(dmul(dmul(x0, x0), q.cp[0]), dmul(dmul(x1, x1), q.cp[1])) <= q.cp[2]) &&
                   (fabs(x1) <= q.cp[3]);
        default:
            return true;
    }
}

__host__ __device__ __forceinline__ uint32_t pack16(uint32_t lo, uint32_t hi) { return lo | (hi << 16); }
__host__ __device__ __forceinline__ uint32_t lo16(uint32_t v) { return v & 0xFFFFu; }
__host__ __device__ __forceinline__ uint32_t hi16(uint32_t v) { return v >> 16; }

// Stored boxes pack one byte per dimension: x | y << 8 | z << 16 | w << 24.
__host__ __device__ __forceinline__ uint32_t pack8(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return a | (b << 8) | (c << 16) | (d << 24);
}

// Fixpoint control block of one instance (device memory).
// 4-byte asynchronous copy global -> shared (cp.async), complete after
// cp_async_wait_all and the group's next barrier.
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---- 1-D bulk copies global -> shared (the TMA engine, no tensor map, no
// multicast) completing on an mbarrier.  Source and destination 16-byte
// aligned, size a multiple of 16 bytes.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of copies completing on the barrier.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(mbar))
                 : "memory");
}

// One bounded probe of the barrier's phase `parity` (the hardware may
// suspend the thread for a while inside the probe).
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t ok = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Probes of a bulk-copy wait before it is given up as failed.
constexpr uint32_t kBulkWaitProbes = 1u << 20;
// FixControl::message of a solve stopped by a device wait that gave up.
constexpr uint32_t kMsgDeviceTimeout = 4;

struct FixControl {
    uint32_t iter;            // iterations completed
    uint32_t stop;            // 1 once a stop rule fired
    uint32_t message;         // GSC_MSG_*
    uint32_t converged;
    uint32_t max_iterations;
    uint32_t stats_cap;       // stats entries (iteration index 1..stats_cap-1)
    uint32_t ticket;          // blocks of the finalize kernel done this iteration
    uint32_t last_new;        // states the last iteration added (saturated at 2^32 - 1)
    unsigned long long candidate_count;
    unsigned long long certified;
    unsigned long long reachable;
    unsigned long long valid_count;
};

}  // namespace gsc_b200
