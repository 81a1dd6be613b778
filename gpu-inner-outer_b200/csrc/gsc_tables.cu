// gsc_tables.cu -- abstraction and query-preparation kernels.
//
// The reference builds one (min_flat, max_flat, valid) triple per (state,
// input) pair in abstraction_kernel (cuda/kernels.cu:164-217), evaluating the
// Euler successor and enumerating every cell of the box.  Here the same boxes
// come from the structure of the unicycle model (model.hpp:26-46): theta
// evolves from (theta cell, omega) alone, v from (v cell, a) alone, x from
// (x, theta, v, input) and y from (y, theta, v, input).  Each coordinate of the
// nominal successor is therefore a per-axis table, bit-identical to the
// reference's per-pair value because it is the same sequence of rounded
// operations.  The box test over cells is a prefix-count (or bit-sliced OR)
// instead of an enumeration.
#include "gsc_kernels.cuh"

namespace gsc_b200 {

namespace {

constexpr int kThreads = 256;

inline unsigned int blocks_for(uint64_t n, int threads = kThreads) {
    uint64_t b = (n + threads - 1) / threads;
    if (b > 0x7FFFFFFFull) b = 0x7FFFFFFFull;
    if (b == 0) b = 1;
    return static_cast<unsigned int>(b);
}

// Blocks of kPlaneThreads threads for one warp per task, at most 16 per SM
// worth of a 148-SM part (the kernels stride over the rest).
inline unsigned int warp_blocks(uint64_t tasks) {
    uint64_t b = (tasks + 7) / 8;
    if (b > 148ull * 16) b = 148ull * 16;
    return static_cast<unsigned int>(b ? b : 1);
}

__device__ __forceinline__ void unflatten(const GridInfo& g, uint64_t s, uint32_t idx[4]) {
    uint64_t r = s / g.n[0];
    idx[0] = static_cast<uint32_t>(s - r * g.n[0]);
    uint64_t r2 = r / g.n[1];
    idx[1] = static_cast<uint32_t>(r - r2 * g.n[1]);
    idx[3] = static_cast<uint32_t>(r2 / g.n[2]);
    idx[2] = static_cast<uint32_t>(r2 - static_cast<uint64_t>(idx[3]) * g.n[2]);
}

__device__ __forceinline__ bool in_rect(const double* lb, const double* ub, const double x[4]) {
    for (int d = 0; d < 4; ++d)
        if (x[d] < lb[d] || x[d] > ub[d]) return false;
    return true;
}

// ---- nominal successors -----------------------------------------------------------------

// One warp per plane (i2, i3, j), plane = (i2*n3 + i3)*M + j; lanes over
// the x then the y cells.  The plane's trajectory terms dt * (v * cos theta)
// and dt * (v * sin theta) do not depend on the cell, so each is computed once
// (staged in shared memory for up to kTermsMax substeps) and added to the
// cell centre in the reference's order (model.hpp:34-45).
constexpr int kPlaneThreads = 256;
constexpr uint32_t kTermsMax = 64;

__global__ void __launch_bounds__(kPlaneThreads) k_nominal_xy(GridInfo g, const double* __restrict__ cosT,
                                                             const double* __restrict__ sinT,
                                                             const double* __restrict__ vseq,
                                                             double* __restrict__ xn, double* __restrict__ yn) {
    __shared__ double terms[kPlaneThreads / 32][2][kTermsMax];
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint64_t planes = static_cast<uint64_t>(g.slices) * g.M;
    const uint64_t wstride = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
    const uint32_t K = g.K;
    const bool staged = K <= kTermsMax;
    for (uint64_t plane = blockIdx.x * static_cast<uint64_t>(blockDim.x >> 5) + wib; plane < planes;
         plane += wstride) {
        const uint32_t j = static_cast<uint32_t>(plane % g.M);
        const uint64_t q = plane / g.M;
        const uint32_t i3 = static_cast<uint32_t>(q % g.n[3]);
        const uint32_t i2 = static_cast<uint32_t>(q / g.n[3]);
        const uint32_t ja = j % g.ma, jw = j / g.ma;
        const double* cs = cosT + static_cast<uint64_t>(i2 * g.mw + jw) * K;
        const double* sn = sinT + static_cast<uint64_t>(i2 * g.mw + jw) * K;
        const double* vs = vseq + static_cast<uint64_t>(i3 * g.ma + ja) * K;
        if (staged) {
            __syncwarp();
            for (uint32_t k = lane; k < K; k += 32) {
                terms[wib][0][k] = dmul(g.dt, dmul(vs[k], cs[k]));
                terms[wib][1][k] = dmul(g.dt, dmul(vs[k], sn[k]));
            }
            __syncwarp();
        }
        for (int axis = 0; axis < 2; ++axis) {
            const uint32_t n = g.n[axis];
            const double* trig = axis ? sn : cs;
            double* out = (axis ? yn : xn) + plane * n;
            for (uint32_t i = lane; i < n; i += 32) {
                double c = centre(g, axis, i);
                if (staged) {
                    for (uint32_t k = 0; k < K; ++k) c = dadd(c, terms[wib][axis][k]);
                } else {
                    for (uint32_t k = 0; k < K; ++k) c = dadd(c, dmul(g.dt, dmul(vs[k], trig[k])));
                }
                out[i] = c;
            }
        }
    }
}

// ---- masks ------------------------------------------------------------------------------

// build_valid_mask / build_candidate_mask (abstraction.hpp:65-106) plus the
// ellipse candidate; counts valid, candidate and candidate-but-invalid cells.
// One warp per x-row (i1, i2, i3); lanes over i0.  The tests on
// dimensions 1-3 (map, obstacles, candidate rectangle) and the y part of the
// candidate ellipse are evaluated once per row; a rectangle test is the AND
// of its per-dimension tests, so the split does not change any result.
__global__ void __launch_bounds__(kPlaneThreads) k_masks(GridInfo g, QueryInfo q, MaskArgs a) {
    unsigned long long nv = 0, nc = 0, nbad = 0, ndiff = 0;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t wstride = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
    const bool few_obstacles = q.n_obstacles <= 32;
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x >> 5) + (threadIdx.x >> 5); r < g.rows;
         r += wstride) {
        const uint32_t i1 = static_cast<uint32_t>(r % g.n[1]);
        const uint64_t r2 = r / g.n[1];
        const uint32_t i2 = static_cast<uint32_t>(r2 % g.n[2]);
        const uint32_t i3 = static_cast<uint32_t>(r2 / g.n[2]);
        double x[4];
        x[1] = centre(g, 1, i1);
        x[2] = centre(g, 2, i2);
        x[3] = centre(g, 3, i3);
        auto in_dims123 = [&](const double* lb, const double* ub) {
            for (int d = 1; d < 4; ++d)
                if (x[d] < lb[d] || x[d] > ub[d]) return false;
            return true;
        };
        const bool map_row = in_dims123(q.map_lb, q.map_ub);
        uint32_t obs_row = 0;
        if (a.build_valid && few_obstacles)
            for (int o = 0; o < q.n_obstacles; ++o)
                if (in_dims123(a.obstacles + 8 * o, a.obstacles + 8 * o + 4)) obs_row |= 1u << o;
        const bool cand_rect_row = q.cand_kind == 0 && in_dims123(q.cand, q.cand + 4);
        const double dy = dsub(x[1], q.cand[1]);
        const double ty = dmul(dmul(dy, dy), q.cand[3]);
        const uint64_t base = r * g.n[0];
        for (uint32_t i0 = lane; i0 < g.n[0]; i0 += 32) {
            const uint64_t s = base + i0;
            x[0] = centre(g, 0, i0);
            bool v;
            if (a.build_valid) {
                v = map_row && !(x[0] < q.map_lb[0] || x[0] > q.map_ub[0]);
                if (v) {
                    if (few_obstacles) {
                        for (uint32_t m = obs_row; m; m &= m - 1) {
                            const int o = __ffs(m) - 1;
                            if (!(x[0] < a.obstacles[8 * o] || x[0] > a.obstacles[8 * o + 4])) {
                                v = false;
                                break;
                            }
                        }
                    } else {
                        for (int o = 0; o < q.n_obstacles; ++o) {
                            if (in_rect(a.obstacles + 8 * o, a.obstacles + 8 * o + 4, x)) {
                                v = false;
                                break;
                            }
                        }
                    }
                }
                // The constraint (abstraction.hpp:96-99): the caller's mask when given
                // (a kCustom predicate evaluated at the centres), else the built-in kind.
                if (v && a.safe)
                    v = (a.safe_rank == 4 ? a.safe[s] : a.safe[static_cast<uint64_t>(i1) * g.n[0] + i0]) != 0;
                else if (v && q.ckind != 0)
                    v = satisfies(q, x[0], x[1]);
                a.valid[s] = v ? 1 : 0;
            } else {
                v = a.valid[s] != 0;
            }
            bool k;
            if (a.build_cand) {
                if (q.cand_kind == 0) {
                    k = cand_rect_row && !(x[0] < q.cand[0] || x[0] > q.cand[4]);
                } else {
                    const double dx = dsub(x[0], q.cand[0]);
                    k = v && (dadd(dmul(dmul(dx, dx), q.cand[2]), ty) <= q.cand[4]);
                }
                a.cand[s] = k ? 1 : 0;
            } else {
                k = a.cand[s] != 0;
            }
            if (a.cmp_safe) {
                const uint8_t sf =
                    a.cmp_rank == 4 ? a.cmp_safe[s] : a.cmp_safe[static_cast<uint64_t>(i1) * g.n[0] + i0];
                ndiff += (v != (sf != 0));
            }
            nv += v;
            nc += k;
            nbad += (k && !v);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        nv += __shfl_down_sync(0xFFFFFFFFu, nv, off);
        nc += __shfl_down_sync(0xFFFFFFFFu, nc, off);
        nbad += __shfl_down_sync(0xFFFFFFFFu, nbad, off);
        ndiff += __shfl_down_sync(0xFFFFFFFFu, ndiff, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nv) atomicAdd(&a.counts[0], nv);
        if (nc) atomicAdd(&a.counts[1], nc);
        if (nbad) atomicAdd(&a.counts[2], nbad);
        if (ndiff) atomicAdd(&a.counts[4], ndiff);
    }
}

// The state constraint at the centres of the (x, y) plane: every built-in
// constraint reads only x and y (config.cpp:62-75).
__global__ void k_safe2(GridInfo g, QueryInfo q, uint8_t* safe2) {
    const uint32_t n = g.n[0] * g.n[1];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t i1 = e / g.n[0];
        const uint32_t i0 = e - i1 * g.n[0];
        safe2[e] = satisfies(q, centre(g, 0, i0), centre(g, 1, i1)) ? 1 : 0;
    }
}

// ---- per-axis boxes ---------------------------------------------------------------------

// x and y boxes: one warp per plane, radius once per plane (it depends on
// the v cell only); theta and v boxes: one thread per entry after that.
__global__ void __launch_bounds__(kPlaneThreads) k_axis_tables(GridInfo g, QueryInfo q,
                                                              const double* __restrict__ xn,
                                                              const double* __restrict__ yn,
                                                              const double* __restrict__ thf,
                                                              const double* __restrict__ vf, uint32_t* xt,
                                                              uint32_t* yt, uint32_t* zt, uint32_t* wt,
                                                              unsigned int* flags) {
    const uint64_t planes = static_cast<uint64_t>(g.slices) * g.M;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t wstride = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
    unsigned int fl = 0;
    for (uint64_t plane = blockIdx.x * static_cast<uint64_t>(blockDim.x >> 5) + (threadIdx.x >> 5);
         plane < planes; plane += wstride) {
        const uint32_t i3 = static_cast<uint32_t>((plane / g.M) % g.n[3]);
        const double vc = centre(g, 3, i3);
        for (int d = 0; d < 2; ++d) {
            const uint32_t n = g.n[d];
            const double r = box_radius(g, q, d, vc);
            const double* nom = (d ? yn : xn) + plane * n;
            uint32_t* out = (d ? yt : xt) + plane * n;
            for (uint32_t i = lane; i < n; i += 32) {
                uint32_t lo, hi;
                const bool ok = axis_box(g, d, nom[i], r, &lo, &hi);
                out[i] = ok ? pack16(lo, hi) : kReject;
                if (ok && hi < lo) fl |= 1u;
                if (ok && hi >= lo && hi - lo >= kBits) fl |= 2u;
            }
        }
    }
    const uint64_t nz = static_cast<uint64_t>(g.n[2]) * g.mw;
    const uint64_t nw = static_cast<uint64_t>(g.n[3]) * g.ma;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < nz + nw;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (e < nz) {
            const uint32_t ee = static_cast<uint32_t>(e);   // i2 * mw + jw
            const double r = box_radius(g, q, 2, 0.0);
            uint32_t lo, hi;
            wrap_box(g, thf[ee], r, &lo, &hi);
            zt[ee] = pack16(lo, hi);
        } else {
            const uint32_t ee = static_cast<uint32_t>(e - nz);   // i3 * ma + ja
            const double r = box_radius(g, q, 3, 0.0);
            uint32_t lo, hi;
            const bool ok = axis_box(g, 3, vf[ee], r, &lo, &hi);
            wt[ee] = ok ? pack16(lo, hi) : kReject;
            if (ok && hi < lo) fl |= 1u;
        }
    }
    if (fl) atomicOr(flags, fl);
}

// ---- bit-sliced sets --------------------------------------------------------------------

// One thread per word: the 32 cells of word w of x-row r.
__global__ void k_pack_bits(GridInfo g, int mode, const uint8_t* __restrict__ src, const uint8_t* __restrict__ src2,
                            bword* __restrict__ out) {
    const uint64_t words = g.rows * g.W;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < words;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t r = e / g.W;
        const uint32_t w = static_cast<uint32_t>(e - r * g.W);
        const uint32_t i1 = static_cast<uint32_t>(r % g.n[1]);
        const uint64_t base = r * g.n[0];
        bword word = 0;
        for (uint32_t b = 0; b < kBits; ++b) {
            const uint32_t i0 = w * kBits + b;
            if (i0 >= g.n[0]) break;
            bool bit;
            switch (mode) {
                case 0: bit = src[base + i0] != 0; break;
                case 1: bit = src[base + i0] == 0; break;
                case 2: bit = src2[i1 * g.n[0] + i0] == 0; break;
                case 3: bit = src[base + i0] != 0 && src2[i1 * g.n[0] + i0] != 0; break;
                default: bit = src[base + i0] != 0 && src2[base + i0] != 0; break;
            }
            word |= static_cast<bword>(bit) << b;
        }
        out[e] = word;
    }
}

__global__ void k_store_words(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t n) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// One warp per x-row.  With fc, the set is the fixpoint's current
// reachable buffer (bits when fc->iter is even, odd otherwise).
__global__ void __launch_bounds__(kPlaneThreads) k_unpack_bits(GridInfo g, const bword* __restrict__ bits,
                                                              uint8_t* __restrict__ out, const FixControl* fc,
                                                              const bword* __restrict__ odd) {
    if (fc && (fc->iter & 1)) bits = odd;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t wstride = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x >> 5) + (threadIdx.x >> 5); r < g.rows;
         r += wstride) {
        const bword* row = bits + r * g.W;
        uint8_t* o = out + r * g.n[0];
        for (uint32_t i0 = lane; i0 < g.n[0]; i0 += 32) o[i0] = static_cast<uint8_t>((row[i0 / kBits] >> (i0 % kBits)) & 1u);
    }
}

// ---- box counts on prefix tables --------------------------------------------------------

// 16-corner inclusion-exclusion of one box [l, r) on a padded int32 table
// (prefix_sum.hpp:65-85): even-popcount corners add.  Exact modulo 2^32.
__device__ __forceinline__ uint32_t count16(const int32_t* __restrict__ P, const GridInfo& g, uint32_t l0,
                                            uint32_t l1, uint32_t l2, uint32_t l3, uint32_t r0, uint32_t r1,
                                            uint32_t r2, uint32_t r3) {
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

// query_box_count (prefix_sum.hpp:87-105): a box crossing the theta seam is split.
__device__ __forceinline__ uint32_t count_box(const int32_t* __restrict__ P, const GridInfo& g, const uint32_t lo[4],
                                              const uint32_t hi[4]) {
    if (lo[2] <= hi[2]) return count16(P, g, lo[0], lo[1], lo[2], lo[3], hi[0] + 1, hi[1] + 1, hi[2] + 1, hi[3] + 1);
    return count16(P, g, lo[0], lo[1], lo[2], lo[3], hi[0] + 1, hi[1] + 1, g.n[2], hi[3] + 1) +
           count16(P, g, lo[0], lo[1], 0, lo[3], hi[0] + 1, hi[1] + 1, hi[2] + 1, hi[3] + 1);
}

// box_satisfies_constraint (abstraction.hpp:108-159) as a count of unsafe
// centres: an empty non-wrap range enumerates no cell and passes.
__device__ __forceinline__ bool box_safe(const GridInfo& g, const uint8_t* __restrict__ safe, int rank,
                                         const int32_t* __restrict__ u2, const int32_t* __restrict__ u4,
                                         const uint32_t lo[4], const uint32_t hi[4]) {
    if (!safe) return true;
    if (hi[0] < lo[0] || hi[1] < lo[1] || hi[3] < lo[3]) return true;
    if (rank == 2) {
        const uint32_t s1 = g.n[0] + 1;
        const uint32_t a = static_cast<uint32_t>(__ldg(u2 + (hi[0] + 1) + (hi[1] + 1) * s1));
        const uint32_t b = static_cast<uint32_t>(__ldg(u2 + lo[0] + (hi[1] + 1) * s1));
        const uint32_t c = static_cast<uint32_t>(__ldg(u2 + (hi[0] + 1) + lo[1] * s1));
        const uint32_t d = static_cast<uint32_t>(__ldg(u2 + lo[0] + lo[1] * s1));
        return a - b - c + d == 0;
    }
    return count_box(u4, g, lo, hi) == 0;
}

struct PairBox {
    bool ok;        // source safe, inside bounds (abstraction validity before the box test)
    uint32_t lo[4], hi[4];
};

__device__ __forceinline__ PairBox pair_box(const GridInfo& g, const uint32_t* __restrict__ xt,
                                            const uint32_t* __restrict__ yt, const uint32_t* __restrict__ zt,
                                            const uint32_t* __restrict__ wt, const uint8_t* __restrict__ safe,
                                            int rank, uint64_t s, uint32_t j) {
    PairBox b;
    uint32_t idx[4];
    unflatten(g, s, idx);
    const uint32_t ja = j % g.ma, jw = j / g.ma;
    const uint64_t plane = (static_cast<uint64_t>(idx[2]) * g.n[3] + idx[3]) * g.M + j;
    const uint32_t xe = __ldg(xt + plane * g.n[0] + idx[0]);
    const uint32_t ye = __ldg(yt + plane * g.n[1] + idx[1]);
    const uint32_t ze = __ldg(zt + idx[2] * g.mw + jw);
    const uint32_t we = __ldg(wt + idx[3] * g.ma + ja);
    bool src = true;
    if (safe) src = (rank == 4) ? safe[s] != 0 : safe[idx[1] * g.n[0] + idx[0]] != 0;
    b.ok = src && xe != kReject && ye != kReject && we != kReject;
    b.lo[0] = lo16(xe);
    b.hi[0] = hi16(xe);
    b.lo[1] = lo16(ye);
    b.hi[1] = hi16(ye);
    b.lo[2] = lo16(ze);
    b.hi[2] = hi16(ze);
    b.lo[3] = lo16(we);
    b.hi[3] = hi16(we);
    return b;
}

// Stored layout: boxes[j * S_pad + s] = {pack8(lo), pack8(hi)} (or, on a
// wide grid, boxes16[j * S + s] = the bounds as 16-bit halves), or the
// sentinel when the pair can never satisfy: abstraction-invalid, or a box
// with no valid cell (the iteration-invariant valid_count == 0 test of
// reachability.hpp:78-84).  A wide entry's first word is lo0 | lo1 << 16
// with lo0 < 65535, so it never equals the sentinel.
__global__ void k_stored_build(GridInfo g, StoredBuildArgs a) {
    const uint64_t rowlen = a.wide ? g.S : a.S_pad;
    const uint64_t total = rowlen * g.M;
    unsigned long long nvp = 0;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t j = static_cast<uint32_t>(e / rowlen);
        const uint64_t s = e - static_cast<uint64_t>(j) * rowlen;
        bool keep = false;
        PairBox b{};
        if (s < g.S) {
            b = pair_box(g, a.xt, a.yt, a.zt, a.wt, a.safe, a.safe_rank, s, j);
            if (b.ok && box_safe(g, a.safe, a.safe_rank, a.unsafe2, a.unsafe4, b.lo, b.hi)) {
                ++nvp;
                keep = count_box(a.pvalid, g, b.lo, b.hi) != 0;
            }
        }
        if (a.wide) {
            a.boxes16[e] = keep ? make_uint4(pack16(b.lo[0], b.lo[1]), pack16(b.lo[2], b.lo[3]),
                                             pack16(b.hi[0], b.hi[1]), pack16(b.hi[2], b.hi[3]))
                                : make_uint4(kBoxSentinel, kBoxSentinel, kBoxSentinel, kBoxSentinel);
        } else {
            a.boxes[e] = keep ? make_uint2(pack8(b.lo[0], b.lo[1], b.lo[2], b.lo[3]),
                                           pack8(b.hi[0], b.hi[1], b.hi[2], b.hi[3]))
                              : make_uint2(kBoxSentinel, kBoxSentinel);
        }
    }
    for (int off = 16; off > 0; off >>= 1) nvp += __shfl_down_sync(0xFFFFFFFFu, nvp, off);
    if ((threadIdx.x & 31) == 0 && nvp) atomicAdd(a.valid_pairs, nvp);
}

__global__ void k_export(GridInfo g, ExportArgs a) {
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < a.pair_count;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t pair = a.pair_begin + e;
        const uint64_t s = pair / g.M;
        const uint32_t j = static_cast<uint32_t>(pair - s * g.M);
        const PairBox b = pair_box(g, a.xt, a.yt, a.zt, a.wt, a.safe, a.safe_rank, s, j);
        const bool v = b.ok && box_safe(g, a.safe, a.safe_rank, a.unsafe2, a.unsafe4, b.lo, b.hi);
        // grid.hpp:22-28 (flatten), x-fastest strides.
        uint32_t mn = 0, mx = 0;
        if (v) {
            mn = b.lo[0] + g.n[0] * (b.lo[1] + g.n[1] * (b.lo[2] + g.n[2] * b.lo[3]));
            mx = b.hi[0] + g.n[0] * (b.hi[1] + g.n[1] * (b.hi[2] + g.n[2] * b.hi[3]));
        }
        a.min_flat[e] = mn;
        a.max_flat[e] = mx;
        a.valid[e] = v ? 1 : 0;
    }
}

// Shift masks of the x boxes of one (slice, input) plane (class_words): a
// state whose box is [i0 + a, i0 + b] is in M_d for every d in [a, b].  A
// box beyond 31 cells of its state, or more than kShiftMax shifts in the
// plane, marks the plane irregular (0xFF), tested state by state.
// One thread per plane; a block first copies its planes' x rows (contiguous)
// into shared memory in one coalesced round, then each thread scans its row
// there twice (a row stride of n0 words): the shift range, then the masks.
__global__ void k_x_classes(GridInfo g, const uint32_t* __restrict__ xt, bword* __restrict__ out) {
    extern __shared__ uint32_t s_xrows[];
    const uint32_t cw = class_words(g);
    const uint32_t n0 = g.n[0];
    const uint64_t planes = static_cast<uint64_t>(g.slices) * g.M;
    for (uint64_t first = blockIdx.x * static_cast<uint64_t>(blockDim.x); first < planes;
         first += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t np = static_cast<uint32_t>(min(static_cast<uint64_t>(blockDim.x), planes - first));
        __syncthreads();   // the previous round's rows are read
        for (uint32_t i = threadIdx.x; i < np * n0; i += blockDim.x) cp_async4(s_xrows + i, xt + first * n0 + i);
        cp_async_wait_all();
        __syncthreads();
        if (threadIdx.x >= np) continue;
        const uint64_t plane = first + threadIdx.x;
        const uint32_t* row = s_xrows + threadIdx.x * n0;
        int dmin = 32, dmax = -32;
        bool irregular = false;
        for (uint32_t i0 = 0; i0 < n0; ++i0) {
            const uint32_t xe = row[i0];
            if (xe == kReject) continue;
            const int a = static_cast<int>(lo16(xe)) - static_cast<int>(i0);
            const int b = static_cast<int>(hi16(xe)) - static_cast<int>(i0);
            if (a < -31 || a > 31 || b < -31 || b > 31 || b < a) {
                irregular = true;
                break;
            }
            dmin = min(dmin, a);
            dmax = max(dmax, b);
        }
        const int nd = (dmax >= dmin) ? dmax - dmin + 1 : 0;
        if (nd > kShiftMax) irregular = true;
        bword* o = out + plane * cw;
        o[0] = irregular ? 0xFFu
                         : static_cast<bword>(nd) |
                               (static_cast<bword>(static_cast<uint8_t>(static_cast<int8_t>(nd ? dmin : 0))) << 8);
        o[1] = o[2] = o[3] = 0;
        // One x word at a time, its masks in registers.
        for (uint32_t w = 0; w < g.W; ++w) {
            bword m[kShiftMax + 1];
#pragma unroll
            for (int k = 0; k <= kShiftMax; ++k) m[k] = 0;
            for (uint32_t i0 = w * kBits; !irregular && i0 < min(n0, (w + 1) * kBits); ++i0) {
                const uint32_t xe = row[i0];
                if (xe == kReject) continue;
                const int a = static_cast<int>(lo16(xe)) - static_cast<int>(i0) - dmin;
                const int b = static_cast<int>(hi16(xe)) - static_cast<int>(i0) - dmin;
                const bword bit = bword(1) << (i0 % kBits);
#pragma unroll
                for (int k = 0; k < kShiftMax; ++k)
                    if (k >= a && k <= b) m[k] |= bit;
                m[kShiftMax] |= bit;
            }
#pragma unroll
            for (int k = 0; k <= kShiftMax; ++k) o[4 + k * g.W + w] = m[k];
        }
    }
}

constexpr int kThreadsReps = 128;

__global__ void k_plane_reps(GridInfo g, const uint32_t* __restrict__ xt, const uint32_t* __restrict__ yt,
                             const uint32_t* __restrict__ wt, uint8_t* __restrict__ rep, uint32_t* max_reps,
                             uint32_t stage_words) {
    // One warp per column; the lanes compare a pair of planes' x and y rows
    // together.  Representatives are kept in increasing order, so an input
    // maps to the lowest earlier input with the same rows and v box.  With
    // stage_words (= ma * (n0 + n1)), the column's x rows and then its y rows
    // are first copied into the warp's shared memory in one round and
    // compared there; else they are compared in global memory.
    extern __shared__ uint32_t s_rows[];
    __shared__ uint8_t s_reps[kThreadsReps / 32][256];
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint8_t* reps = s_reps[wib];
    uint32_t* rows = s_rows + static_cast<uint64_t>(wib) * stage_words;
    const uint32_t n0 = g.n[0], n1 = g.n[1], ma = g.ma;
    const uint32_t nx = ma * n0;
    const uint64_t columns = static_cast<uint64_t>(g.slices) * g.mw;
    const uint64_t wstride = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
    uint32_t most = 0;
    for (uint64_t col = blockIdx.x * static_cast<uint64_t>(blockDim.x >> 5) + wib; col < columns; col += wstride) {
        // Planes are ((i2 * n3 + i3) * M + j) with j = ja + ma * jw, so column
        // col = (i2 * n3 + i3) * mw + jw starts at plane col * ma.
        const uint32_t i3 = static_cast<uint32_t>((col / g.mw) % g.n[3]);
        const uint64_t p0 = col * ma;
        const uint32_t* X = xt + p0 * n0;
        const uint32_t* Y = yt + p0 * n1;
        if (stage_words) {
            for (uint32_t i = lane; i < nx; i += 32) cp_async4(rows + i, X + i);
            for (uint32_t i = lane; i < ma * n1; i += 32) cp_async4(rows + nx + i, Y + i);
            cp_async_wait_all();
            __syncwarp();
            X = rows;
            Y = rows + nx;
        }
        uint32_t nrep = 0;
        for (uint32_t ja = 0; ja < ma; ++ja) {
            const uint32_t we = wt[i3 * ma + ja];
            uint32_t r = ja;
            for (uint32_t k = 0; k < nrep; ++k) {
                const uint32_t jb = reps[k];
                if (wt[i3 * ma + jb] != we) continue;
                bool same = true;
                for (uint32_t i = lane; i < n0; i += 32) same = same && X[jb * n0 + i] == X[ja * n0 + i];
                for (uint32_t i = lane; i < n1; i += 32) same = same && Y[jb * n1 + i] == Y[ja * n1 + i];
                if (__all_sync(0xFFFFFFFFu, same)) {
                    r = jb;
                    break;
                }
            }
            if (r == ja) {
                if (lane == 0) reps[nrep] = static_cast<uint8_t>(ja);
                ++nrep;
            }
            if (lane == 0) rep[p0 + ja] = static_cast<uint8_t>(r);
            __syncwarp();
        }
        most = max(most, nrep);
    }
    if (lane == 0 && most) atomicMax(max_reps, most);
}

// 2-D prefix of unsafe (x, y) centres; one block: rows, then columns.
__global__ void k_prefix2(GridInfo g, const uint8_t* __restrict__ safe2, int32_t* __restrict__ t) {
    const uint32_t s1 = g.n[0] + 1;
    for (uint32_t y = threadIdx.x; y <= g.n[1]; y += blockDim.x) {
        int32_t acc = 0;
        t[y * s1] = 0;
        for (uint32_t x = 1; x <= g.n[0]; ++x) {
            if (y > 0) acc += safe2[(y - 1) * g.n[0] + (x - 1)] == 0;
            t[y * s1 + x] = acc;
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x <= g.n[0]; x += blockDim.x) {
        int32_t acc = 0;
        for (uint32_t y = 1; y <= g.n[1]; ++y) {
            acc += t[y * s1 + x];
            t[y * s1 + x] = acc;
        }
    }
}

}  // namespace

cudaError_t launch_nominal_xy(const GridInfo& g, const double* cosT, const double* sinT, const double* vseq,
                              double* xn, double* yn, cudaStream_t st) {
    k_nominal_xy<<<warp_blocks(static_cast<uint64_t>(g.slices) * g.M), kPlaneThreads, 0, st>>>(g, cosT, sinT, vseq,
                                                                                            xn, yn);
    return cudaGetLastError();
}

cudaError_t launch_masks(const GridInfo& g, const QueryInfo& q, const MaskArgs& a, cudaStream_t st) {
    k_masks<<<warp_blocks(g.rows), kPlaneThreads, 0, st>>>(g, q, a);
    return cudaGetLastError();
}

cudaError_t launch_safe2(const GridInfo& g, const QueryInfo& q, uint8_t* safe2, cudaStream_t st) {
    k_safe2<<<blocks_for(static_cast<uint64_t>(g.n[0]) * g.n[1]), kThreads, 0, st>>>(g, q, safe2);
    return cudaGetLastError();
}

cudaError_t launch_axis_tables(const GridInfo& g, const QueryInfo& q, const double* xn, const double* yn,
                               const double* thf, const double* vf, uint32_t* xt, uint32_t* yt, uint32_t* zt,
                               uint32_t* wt, unsigned int* flags, cudaStream_t st) {
    k_axis_tables<<<warp_blocks(static_cast<uint64_t>(g.slices) * g.M), kPlaneThreads, 0, st>>>(g, q, xn, yn, thf,
                                                                                             vf, xt, yt, zt, wt,
                                                                                             flags);
    return cudaGetLastError();
}

cudaError_t launch_pack_bits(const GridInfo& g, int mode, const uint8_t* src, const uint8_t* src2, bword* out,
                             cudaStream_t st) {
    k_pack_bits<<<blocks_for(g.rows * g.W), kThreads, 0, st>>>(g, mode, src, src2, out);
    return cudaGetLastError();
}

cudaError_t launch_unpack_bits(const GridInfo& g, const bword* bits, uint8_t* out, cudaStream_t st) {
    k_unpack_bits<<<warp_blocks(g.rows), kPlaneThreads, 0, st>>>(g, bits, out, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_store_words(const uint32_t* src, uint32_t* dst, uint32_t n, cudaStream_t st) {
    k_store_words<<<1, 32, 0, st>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_unpack_reach(const GridInfo& g, const FixControl* fc, const bword* reach0, const bword* reach1,
                                uint8_t* out, cudaStream_t st) {
    k_unpack_bits<<<warp_blocks(g.rows), kPlaneThreads, 0, st>>>(g, reach0, out, fc, reach1);
    return cudaGetLastError();
}

cudaError_t launch_prefix2_unsafe(const GridInfo& g, const uint8_t* safe2, int32_t* table, cudaStream_t st) {
    k_prefix2<<<1, 256, 0, st>>>(g, safe2, table);
    return cudaGetLastError();
}

cudaError_t launch_stored_build(const GridInfo& g, const StoredBuildArgs& a, cudaStream_t st) {
    k_stored_build<<<blocks_for((a.wide ? g.S : a.S_pad) * g.M), kThreads, 0, st>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_x_classes(const GridInfo& g, const uint32_t* xt, bword* xcls, cudaStream_t st) {
    // Threads (planes) a block: as many rows as fit 44 KB of shared memory, 32 to 128.
    uint32_t tpb = static_cast<uint32_t>((44u * 1024u) / (4u * std::max<uint32_t>(g.n[0], 1u)));
    tpb = std::min<uint32_t>(128u, std::max<uint32_t>(32u, tpb & ~31u));
    if (4ull * tpb * g.n[0] > 48 * 1024) return cudaErrorInvalidValue;
    k_x_classes<<<blocks_for(static_cast<uint64_t>(g.slices) * g.M, tpb), tpb, 4ull * tpb * g.n[0], st>>>(g, xt, xcls);
    return cudaGetLastError();
}

cudaError_t launch_plane_reps(const GridInfo& g, const uint32_t* xt, const uint32_t* yt, const uint32_t* wt,
                              uint8_t* xrep, uint32_t* max_reps, cudaStream_t st) {
    const uint64_t warps = static_cast<uint64_t>(g.slices) * g.mw;
    uint64_t b = (warps + kThreadsReps / 32 - 1) / (kThreadsReps / 32);
    if (b > 8192) b = 8192;
    // Stage a column's rows in shared memory when they fit 44 KB a block (the
    // default 48 KB less the representatives' static arrays).
    const uint64_t words = static_cast<uint64_t>(g.ma) * (g.n[0] + g.n[1]);
    const uint32_t stage = words * 4 * (kThreadsReps / 32) <= 44 * 1024 ? static_cast<uint32_t>(words) : 0u;
    k_plane_reps<<<static_cast<unsigned int>(b), kThreadsReps, 4ull * stage * (kThreadsReps / 32), st>>>(
        g, xt, yt, wt, xrep, max_reps, stage);
    return cudaGetLastError();
}

cudaError_t launch_export(const GridInfo& g, const ExportArgs& a, cudaStream_t st) {
    k_export<<<blocks_for(a.pair_count), kThreads, 0, st>>>(g, a);
    return cudaGetLastError();
}

}  // namespace gsc_b200
