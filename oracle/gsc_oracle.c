/*
 * gsc_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see gsc_oracle.h).
 *
 * A plain-C restatement of the reference CPU method of zzx-ur/gpu-inner-outer.
 * Floating-point expressions keep the reference's operation order and are
 * compiled without contraction (-ffp-contract=off), so every successor box is
 * bit-identical to the reference's.  OpenMP only splits independent states;
 * it never changes an arithmetic result.
 */
#include "gsc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    double lb[4], ub[4], eta[4];
    uint32_t shape[4];
    uint64_t strides[4];
    uint64_t total;
    int wrap_dim;
} grid4;

typedef struct {
    double lb[2], eta[2];
    uint32_t shape[2];
    uint64_t total;
} grid2;

static double now_ms(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec * 1e-6;
}

/* grid.hpp:103-141 (build_state_grid) and grid.hpp:143-168 (build_input_grid). */
static int make_grids(const orc_case* c, grid4* g, grid2* u) {
    g->wrap_dim = c->wrap_dim;
    g->total = 1;
    for (int d = 0; d < 4; ++d) {
        g->lb[d] = c->state_lb[d];
        g->ub[d] = c->state_ub[d];
        g->eta[d] = c->state_eta[d];
        if (!(c->state_eta[d] > 0.0)) return -1;
        const double width = c->state_ub[d] - c->state_lb[d];
        if (!(width > 0.0)) return -1;
        g->shape[d] = (uint32_t)ceil(width / c->state_eta[d]);
    }
    g->strides[0] = 1;
    for (int d = 1; d < 4; ++d) g->strides[d] = g->strides[d - 1] * g->shape[d - 1];
    for (int d = 0; d < 4; ++d) g->total *= g->shape[d];
    if (g->total > 0xFFFFFFFFull) return -1;   /* StateIndex = uint32_t */
    for (int d = 0; d < 2; ++d) {
        u->lb[d] = c->input_lb[d];
        u->eta[d] = c->input_eta[d];
        if (!(c->input_eta[d] > 0.0)) return -1;
        const double width = c->input_ub[d] - c->input_lb[d];
        if (!(width > 0.0)) return -1;
        u->shape[d] = (uint32_t)ceil(width / c->input_eta[d]);
    }
    u->total = (uint64_t)u->shape[0] * u->shape[1];
    return 0;
}

int orc_shapes(const orc_case* c, uint32_t shape[4], uint32_t input_shape[2]) {
    grid4 g;
    grid2 u;
    if (make_grids(c, &g, &u) != 0) return -1;
    for (int d = 0; d < 4; ++d) shape[d] = g.shape[d];
    input_shape[0] = u.shape[0];
    input_shape[1] = u.shape[1];
    return 0;
}

/* grid.hpp:30-36 (unflatten) and grid.hpp:38-44 (center). */
static void unflatten(const grid4* g, uint64_t flat, uint32_t idx[4]) {
    uint64_t v = flat;
    for (int d = 3; d >= 0; --d) {
        idx[d] = (uint32_t)(v / g->strides[d]);
        v %= g->strides[d];
    }
}

static uint64_t flatten(const grid4* g, const uint32_t idx[4]) {
    return (uint64_t)idx[0] * g->strides[0] + (uint64_t)idx[1] * g->strides[1] +
           (uint64_t)idx[2] * g->strides[2] + (uint64_t)idx[3] * g->strides[3];
}

static void center(const grid4* g, uint64_t flat, double out[4]) {
    uint32_t idx[4];
    unflatten(g, flat, idx);
    for (int d = 0; d < 4; ++d) out[d] = g->lb[d] + ((double)idx[d] + 0.5) * g->eta[d];
}

/* grid.hpp:68-78: input flat = i0 + shape0 * i1. */
static void input_center(const grid2* u, uint64_t flat, double out[2]) {
    uint32_t idx[2];
    idx[1] = (uint32_t)(flat / u->shape[0]);
    idx[0] = (uint32_t)(flat % u->shape[0]);
    for (int d = 0; d < 2; ++d) out[d] = u->lb[d] + ((double)idx[d] + 0.5) * u->eta[d];
}

/* config.cpp:62-75 (hyperbolic, elliptic) and the quadric custom predicate;
 * satisfies_state_constraint config.cpp:108-127. */
static int satisfies(const orc_case* c, const double x[4]) {
    switch (c->constraint_kind) {
        case ORC_CONSTRAINT_NONE:
            return 1;
        case ORC_CONSTRAINT_HYPERBOLIC: {
            const double x1_sq = x[0] * x[0];
            const double x2_sq = x[1] * x[1];
            return (x1_sq - x2_sq <= c->cparam[0]) && (c->cparam[1] * x2_sq - x1_sq <= c->cparam[2]);
        }
        case ORC_CONSTRAINT_ELLIPTIC: {
            const double t1 = (x[0] / c->cparam[0]) * (x[0] / c->cparam[0]);
            const double t2 = (x[1] / c->cparam[1]) * (x[1] / c->cparam[1]);
            return t1 + t2 <= 1.0;
        }
        case ORC_CONSTRAINT_QUADRIC:
            return ((x[0] * x[0]) * c->cparam[0] - (x[1] * x[1]) * c->cparam[1] <= c->cparam[2]) &&
                   (fabs(x[1]) <= c->cparam[3]);
        default:
            return 1;
    }
}

/* config.cpp:80-87. */
static int point_in_rect(const double lb[4], const double ub[4], const double x[4]) {
    for (int d = 0; d < 4; ++d)
        if (x[d] < lb[d] || x[d] > ub[d]) return 0;
    return 1;
}

/* model.hpp:14-24. */
static double wrap_angle(double x) {
    const double kPi = 3.14159265358979323846;
    const double kTwoPi = 2.0 * kPi;
    while (x < -kPi) x += kTwoPi;
    while (x >= kPi) x -= kTwoPi;
    return x;
}

/* model.hpp:91-112 with nominal_step :26-46, jacobian_x_times_half_eta :55-76,
 * jacobian_w_times_half_disturbance :84-89. */
static void successor_box(const orc_case* c, const double x[4], const double u[2],
                          const double eta[4], double mn[4], double mx[4]) {
    double out[4] = {x[0], x[1], x[2], x[3]};
    const double dt = c->sample_time / (double)c->substeps;
    for (uint32_t s = 0; s < c->substeps; ++s) {
        const double dx = out[3] * cos(out[2]);
        const double dy = out[3] * sin(out[2]);
        const double dtheta = u[1];
        const double dv = u[0];
        out[0] += dt * dx;
        out[1] += dt * dy;
        out[2] = wrap_angle(out[2] + dt * dtheta);
        out[3] += dt * dv;
    }
    const double T = c->sample_time;
    const double half_eta[4] = {0.5 * eta[0], 0.5 * eta[1], 0.5 * eta[2], 0.5 * eta[3]};
    const double abs_v = fabs(x[3]);
    double jfx[4], jfw[4];
    jfx[0] = half_eta[0] + T * abs_v * half_eta[2] + T * half_eta[3];
    jfx[1] = half_eta[1] + T * abs_v * half_eta[2] + T * half_eta[3];
    jfx[2] = half_eta[2];
    jfx[3] = half_eta[3];
    for (int d = 0; d < 4; ++d) jfw[d] = T * c->dhw[d];
    for (int d = 0; d < 4; ++d) {
        const double radius = jfx[d] + jfw[d];
        mn[d] = out[d] - radius;
        mx[d] = out[d] + radius;
    }
}

/* grid.hpp:46-57 (wrap_value). */
static double wrap_value(const grid4* g, double x) {
    const double low = g->lb[g->wrap_dim];
    const double high = g->ub[g->wrap_dim];
    const double span = high - low;
    while (x < low) x += span;
    while (x >= high) x -= span;
    return x;
}

static void quantise_dim(const grid4* g, int d, double lo_c, double hi_c, uint32_t* lo, uint32_t* hi) {
    int64_t lower = (int64_t)floor((lo_c - g->lb[d]) / g->eta[d]);
    int64_t upper = (int64_t)ceil((hi_c - g->lb[d]) / g->eta[d]) - 1;
    if (lower < 0) lower = 0;
    if (upper < 0) upper = 0;
    if (lower >= (int64_t)g->shape[d]) lower = (int64_t)g->shape[d] - 1;
    if (upper >= (int64_t)g->shape[d]) upper = (int64_t)g->shape[d] - 1;
    *lo = (uint32_t)lower;
    *hi = (uint32_t)upper;
}

/* grid.hpp:181-251 (continuous_box_to_index_box).  Returns 0 when rejected. */
static int to_index_box(const grid4* g, const double mn[4], const double mx[4],
                        uint32_t bmin[4], uint32_t bmax[4]) {
    const double kEps = 1e-9;
    for (int d = 0; d < 4; ++d) {
        if (d == g->wrap_dim) continue;
        if (mn[d] < g->lb[d] - kEps || mx[d] > g->ub[d] + kEps) return 0;
    }
    const int w = g->wrap_dim;
    const double wrap_span = g->ub[w] - g->lb[w];
    const double raw_wrap_width = mx[w] - mn[w];
    for (int d = 0; d < 4; ++d) {
        if (d == w) {
            if (raw_wrap_width >= wrap_span - kEps) {
                bmin[d] = 0;
                bmax[d] = g->shape[d] - 1;
                continue;
            }
            quantise_dim(g, d, wrap_value(g, mn[d]), wrap_value(g, mx[d]), &bmin[d], &bmax[d]);
            continue;
        }
        quantise_dim(g, d, mn[d], mx[d], &bmin[d], &bmax[d]);
    }
    return 1;
}

/* abstraction.hpp:108-159 (box_satisfies_constraint), loop structure kept. */
static int box_safe(const orc_case* c, const grid4* g, const uint32_t bmin[4], const uint32_t bmax[4]) {
    if (c->constraint_kind == ORC_CONSTRAINT_NONE) return 1;
    const int wrap_dim = g->wrap_dim;
    const int has_wrap = bmin[wrap_dim] > bmax[wrap_dim];
    uint32_t idx[4];
    for (idx[3] = bmin[3]; idx[3] <= bmax[3]; ++idx[3]) {
        for (idx[2] = bmin[2];; ++idx[2]) {
            int in_range_2;
            if (wrap_dim == 2 && has_wrap)
                in_range_2 = (idx[2] >= bmin[2] || idx[2] <= bmax[2]);
            else
                in_range_2 = (idx[2] <= bmax[2]);
            if (!in_range_2 && idx[2] > bmax[2] && (!has_wrap || idx[2] >= g->shape[2])) break;
            for (idx[1] = bmin[1]; idx[1] <= bmax[1]; ++idx[1]) {
                for (idx[0] = bmin[0]; idx[0] <= bmax[0]; ++idx[0]) {
                    double ctr[4];
                    center(g, flatten(g, idx), ctr);
                    if (!satisfies(c, ctr)) return 0;
                }
            }
            if (wrap_dim == 2 && has_wrap && idx[2] == g->shape[2] - 1)
                idx[2] = (uint32_t)-1;
            else if (idx[2] == bmax[2])
                break;
        }
    }
    return 1;
}

/* abstraction.hpp:65-106 plus the ellipse candidate. */
static int build_masks(const orc_case* c, const grid4* g, uint8_t* valid, uint8_t* cand) {
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (uint64_t f = 0; f < g->total; ++f) {
        double x[4];
        center(g, f, x);
        int v = point_in_rect(c->map_lb, c->map_ub, x);
        if (v) {
            for (int o = 0; o < c->n_obstacles; ++o) {
                if (point_in_rect(c->obstacles[o], c->obstacles[o] + 4, x)) {
                    v = 0;
                    break;
                }
            }
        }
        if (v && c->constraint_kind != ORC_CONSTRAINT_NONE) v = satisfies(c, x);
        valid[f] = (uint8_t)(v ? 1 : 0);
        int k;
        if (c->candidate_kind == ORC_CANDIDATE_RECT) {
            k = point_in_rect(c->cand, c->cand + 4, x);
        } else {
            const double dx = x[0] - c->cand[0];
            const double dy = x[1] - c->cand[1];
            k = v && ((dx * dx) * c->cand[2] + (dy * dy) * c->cand[3] <= c->cand[4]);
        }
        cand[f] = (uint8_t)(k ? 1 : 0);
        if (k && !v) bad = 1;
    }
    return bad ? -1 : 0;
}

int orc_masks(const orc_case* c, uint8_t* valid, uint8_t* candidate) {
    grid4 g;
    grid2 u;
    if (make_grids(c, &g, &u) != 0) return -2;
    return build_masks(c, &g, valid, candidate);
}

/* One state's row of the abstraction (abstraction.hpp:168-208). */
static uint64_t abstraction_row(const orc_case* c, const grid4* g, const grid2* u, uint64_t s,
                                uint32_t* mnf, uint32_t* mxf, uint8_t* pv) {
    uint64_t nvalid = 0;
    double x[4];
    center(g, s, x);
    for (uint64_t j = 0; j < u->total; ++j) {
        mnf[j] = 0;
        mxf[j] = 0;
        pv[j] = 0;
    }
    if (c->constraint_kind != ORC_CONSTRAINT_NONE && !satisfies(c, x)) return 0;
    for (uint64_t j = 0; j < u->total; ++j) {
        double uc[2], mn[4], mx[4];
        uint32_t bmin[4], bmax[4];
        input_center(u, j, uc);
        successor_box(c, x, uc, g->eta, mn, mx);
        if (!to_index_box(g, mn, mx, bmin, bmax)) continue;
        if (!box_safe(c, g, bmin, bmax)) continue;
        mnf[j] = (uint32_t)flatten(g, bmin);
        mxf[j] = (uint32_t)flatten(g, bmax);
        pv[j] = 1;
        ++nvalid;
    }
    return nvalid;
}

static int set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    return 0;
}

int orc_abstraction(const orc_case* c, uint32_t* min_flat, uint32_t* max_flat, uint8_t* pair_valid,
                    int nthreads) {
    grid4 g;
    grid2 u;
    if (make_grids(c, &g, &u) != 0) return -2;
    set_threads(nthreads);
    const uint64_t M = u.total;
#pragma omp parallel for schedule(dynamic, 64)
    for (uint64_t s = 0; s < g.total; ++s)
        abstraction_row(c, &g, &u, s, min_flat + s * M, max_flat + s * M, pair_valid + s * M);
    return 0;
}

/* grid.hpp:253-269 (build_prefix_layout). */
static void prefix_layout(const uint32_t shape[4], uint64_t pstride[4], uint64_t* total) {
    pstride[0] = 1;
    for (int d = 1; d < 4; ++d) pstride[d] = pstride[d - 1] * (shape[d - 1] + 1);
    *total = pstride[3] * (shape[3] + 1);
}

/* prefix_sum.hpp:15-63.  The 16-term recurrence is restated as four
 * successive one-axis running sums, which yields the same table entry for
 * entry in exact u64 arithmetic. */
void orc_prefix(const uint32_t shape[4], const uint8_t* mask, uint64_t* out) {
    uint64_t ps[4], total;
    prefix_layout(shape, ps, &total);
    memset(out, 0, total * sizeof(uint64_t));
    const uint64_t n0 = shape[0], n1 = shape[1], n2 = shape[2], n3 = shape[3];
    for (uint64_t w = 0; w < n3; ++w)
        for (uint64_t z = 0; z < n2; ++z)
            for (uint64_t y = 0; y < n1; ++y)
                for (uint64_t x = 0; x < n0; ++x) {
                    const uint64_t flat = x + n0 * (y + n1 * (z + n2 * w));
                    out[(x + 1) + (y + 1) * ps[1] + (z + 1) * ps[2] + (w + 1) * ps[3]] = mask[flat] ? 1 : 0;
                }
    for (int d = 0; d < 4; ++d) {
        const uint64_t len = shape[d] + 1;
        const uint64_t st = ps[d];
        for (uint64_t base = 0; base < total; ++base) {
            if ((base / st) % len != 0) continue;   /* start of a line along d */
            for (uint64_t k = 1; k < len; ++k) out[base + k * st] += out[base + (k - 1) * st];
        }
    }
}

/* prefix_sum.hpp:65-85 (query_box_single): even-popcount corners add. */
static uint64_t query_single(const uint64_t ps[4], const uint64_t* data, const uint32_t bmin[4],
                             const uint32_t bmax[4]) {
    const uint32_t l[4] = {bmin[0], bmin[1], bmin[2], bmin[3]};
    const uint32_t r[4] = {bmax[0] + 1, bmax[1] + 1, bmax[2] + 1, bmax[3] + 1};
    uint64_t total = 0;
    for (int m = 0; m < 16; ++m) {
        const uint64_t x0 = (m & 1) ? l[0] : r[0];
        const uint64_t x1 = (m & 2) ? l[1] : r[1];
        const uint64_t x2 = (m & 4) ? l[2] : r[2];
        const uint64_t x3 = (m & 8) ? l[3] : r[3];
        const uint64_t v = data[x0 * ps[0] + x1 * ps[1] + x2 * ps[2] + x3 * ps[3]];
        if ((__builtin_popcount((unsigned)m) & 1) == 0)
            total += v;
        else
            total -= v;
    }
    return total;
}

/* prefix_sum.hpp:87-105 (query_box_count): a wrapped box is split in two. */
static uint64_t query_count(const grid4* g, const uint64_t ps[4], const uint64_t* data,
                            uint32_t min_flat, uint32_t max_flat) {
    uint32_t bmin[4], bmax[4];
    unflatten(g, min_flat, bmin);
    unflatten(g, max_flat, bmax);
    const int w = g->wrap_dim;
    if (bmin[w] <= bmax[w]) return query_single(ps, data, bmin, bmax);
    uint32_t lmax[4] = {bmax[0], bmax[1], bmax[2], bmax[3]};
    uint32_t rmin[4] = {bmin[0], bmin[1], bmin[2], bmin[3]};
    lmax[w] = g->shape[w] - 1;
    rmin[w] = 0;
    return query_single(ps, data, bmin, lmax) + query_single(ps, data, rmin, bmax);
}

uint64_t orc_query(const uint32_t shape[4], int wrap_dim, const uint64_t* prefix, uint32_t min_flat,
                   uint32_t max_flat) {
    grid4 g;
    memset(&g, 0, sizeof(g));
    g.wrap_dim = wrap_dim;
    g.strides[0] = 1;
    for (int d = 0; d < 4; ++d) g.shape[d] = shape[d];
    for (int d = 1; d < 4; ++d) g.strides[d] = g.strides[d - 1] * shape[d - 1];
    uint64_t ps[4], total;
    prefix_layout(shape, ps, &total);
    return query_count(&g, ps, prefix, min_flat, max_flat);
}

/* The per-state body of one Jacobi iteration (reachability.hpp:59-109).
 * Returns 1 if the state was processed and satisfied, with the chosen input. */
static int state_step(const grid4* g, uint64_t M, const uint64_t ps[4], const uint64_t* pre_valid,
                      const uint64_t* pre_reach, const uint32_t* mnf, const uint32_t* mxf,
                      const uint8_t* pv, uint32_t* chosen) {
    for (uint64_t j = 0; j < M; ++j) {
        if (!pv[j]) continue;
        const uint64_t vc = query_count(g, ps, pre_valid, mnf[j], mxf[j]);
        if (vc == 0) continue;
        const uint64_t rc = query_count(g, ps, pre_reach, mnf[j], mxf[j]);
        if (rc == vc) {
            *chosen = (uint32_t)j;
            return 1;
        }
    }
    return 0;
}

int orc_solve(const orc_case* c, uint8_t* valid_out, uint8_t* cand_out, uint8_t* reach_out,
              uint32_t* ctl_out, uint32_t* step_out, uint64_t* iter_new_reach, uint64_t* iter_new_cert,
              uint32_t iter_cap, orc_summary* sm, int nthreads) {
    grid4 g;
    grid2 u;
    if (make_grids(c, &g, &u) != 0) return -2;
    set_threads(nthreads);
    const uint64_t S = g.total, M = u.total, P = S * M;
    uint8_t* valid = (uint8_t*)malloc(S);
    uint8_t* cand = (uint8_t*)malloc(S);
    uint8_t* reach = (uint8_t*)malloc(S);
    uint8_t* reach_next = (uint8_t*)malloc(S);
    uint32_t* ctl = (uint32_t*)malloc(S * sizeof(uint32_t));
    uint32_t* step = (uint32_t*)malloc(S * sizeof(uint32_t));
    uint32_t* mnf = (uint32_t*)malloc(P * sizeof(uint32_t));
    uint32_t* mxf = (uint32_t*)malloc(P * sizeof(uint32_t));
    uint8_t* pv = (uint8_t*)malloc(P);
    uint64_t ps[4], T;
    prefix_layout(g.shape, ps, &T);
    uint64_t* pre_valid = (uint64_t*)malloc(T * sizeof(uint64_t));
    uint64_t* pre_reach = (uint64_t*)malloc(T * sizeof(uint64_t));
    int rc = 0;
    if (!valid || !cand || !reach || !reach_next || !ctl || !step || !mnf || !mxf || !pv || !pre_valid ||
        !pre_reach) {
        rc = -3;
        goto done;
    }
    /* prepare_case_cpu, abstraction.hpp:276-307. */
    if (build_masks(c, &g, valid, cand) != 0) {
        rc = -1;
        goto done;
    }
    double t0 = now_ms();
    uint64_t valid_pairs = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : valid_pairs)
    for (uint64_t s = 0; s < S; ++s) valid_pairs += abstraction_row(c, &g, &u, s, mnf + s * M, mxf + s * M, pv + s * M);
    double t1 = now_ms();

    /* solve_backward_cpu, reachability.hpp:30-155. */
    uint64_t candidate_count = 0, valid_count = 0;
    for (uint64_t i = 0; i < S; ++i) {
        reach[i] = cand[i];
        ctl[i] = 0xFFFFFFFFu;
        step[i] = 0xFFFFFFFFu;
        if (cand[i]) {
            step[i] = 0;
            ++candidate_count;
        }
        valid_count += valid[i] ? 1 : 0;
    }
    orc_prefix(g.shape, valid, pre_valid);
    uint64_t certified = 0;
    uint32_t iterations = 0;
    int converged = 0, message = ORC_MSG_NONE;
    double t2 = now_ms();
    for (uint32_t iter = 1; iter <= c->max_iterations; ++iter) {
        orc_prefix(g.shape, reach, pre_reach);
        memcpy(reach_next, reach, S);
        uint64_t new_reach = 0, new_cert = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : new_reach, new_cert)
        for (uint64_t s = 0; s < S; ++s) {
            if (!valid[s]) continue;
            const int is_cand = cand[s] != 0;
            const int already_reached = reach[s] != 0;
            const int already_cert = ctl[s] != 0xFFFFFFFFu;
            if ((!is_cand && already_reached) || (is_cand && already_cert)) continue;
            uint32_t chosen;
            if (!state_step(&g, M, ps, pre_valid, pre_reach, mnf + s * M, mxf + s * M, pv + s * M, &chosen))
                continue;
            if (!already_reached) {
                reach_next[s] = 1;
                ++new_reach;
            }
            if (!already_cert) {
                ctl[s] = chosen;
                if (is_cand)
                    ++new_cert;
                else
                    step[s] = iter;
            }
        }
        memcpy(reach, reach_next, S);
        certified += new_cert;
        iterations = iter;
        if (iter_new_reach && iter <= iter_cap) iter_new_reach[iter - 1] = new_reach;
        if (iter_new_cert && iter <= iter_cap) iter_new_cert[iter - 1] = new_cert;
        if (certified == candidate_count) {
            converged = 1;
            message = ORC_MSG_CONVERGED;
            break;
        }
        if (new_reach == 0 && new_cert == 0) {
            message = ORC_MSG_STALLED;
            break;
        }
    }
    double t3 = now_ms();
    if (!converged && message == ORC_MSG_NONE) message = ORC_MSG_MAX_ITER;
    uint64_t reachable_states = 0;
    for (uint64_t i = 0; i < S; ++i) reachable_states += reach[i] == 1;

    if (sm) {
        memset(sm, 0, sizeof(*sm));
        for (int d = 0; d < 4; ++d) sm->shape[d] = g.shape[d];
        sm->input_shape[0] = u.shape[0];
        sm->input_shape[1] = u.shape[1];
        sm->states = S;
        sm->inputs = M;
        sm->pairs = P;
        sm->iterations = iterations;
        sm->converged = converged;
        sm->message = message;
        sm->reachable_states = reachable_states;
        sm->certified_candidates = certified;
        sm->candidate_count = candidate_count;
        sm->valid_count = valid_count;
        sm->valid_pairs = valid_pairs;
        sm->abstraction_ms = t1 - t0;
        sm->solve_ms = t3 - t2;
    }
    if (valid_out) memcpy(valid_out, valid, S);
    if (cand_out) memcpy(cand_out, cand, S);
    if (reach_out) memcpy(reach_out, reach, S);
    if (ctl_out) memcpy(ctl_out, ctl, S * sizeof(uint32_t));
    if (step_out) memcpy(step_out, step, S * sizeof(uint32_t));
done:
    free(valid);
    free(cand);
    free(reach);
    free(reach_next);
    free(ctl);
    free(step);
    free(mnf);
    free(mxf);
    free(pv);
    free(pre_valid);
    free(pre_reach);
    return rc;
}

int orc_spot_step(const orc_case* c, const uint8_t* valid, const uint8_t* cand, const uint8_t* reach_prev,
                  const uint32_t* ctl_prev, const uint32_t* step_prev, uint32_t iter, const uint64_t* states,
                  uint64_t n_states, uint8_t* reach_next_out, uint32_t* ctl_out, uint32_t* step_out,
                  int nthreads) {
    grid4 g;
    grid2 u;
    if (make_grids(c, &g, &u) != 0) return -2;
    set_threads(nthreads);
    const uint64_t M = u.total;
    uint64_t ps[4], T;
    prefix_layout(g.shape, ps, &T);
    uint64_t* pre_valid = (uint64_t*)malloc(T * sizeof(uint64_t));
    uint64_t* pre_reach = (uint64_t*)malloc(T * sizeof(uint64_t));
    if (!pre_valid || !pre_reach) {
        free(pre_valid);
        free(pre_reach);
        return -3;
    }
    orc_prefix(g.shape, valid, pre_valid);
    orc_prefix(g.shape, reach_prev, pre_reach);
    int bad = 0;
#pragma omp parallel reduction(| : bad)
    {
        uint32_t* mnf = (uint32_t*)malloc(M * sizeof(uint32_t));
        uint32_t* mxf = (uint32_t*)malloc(M * sizeof(uint32_t));
        uint8_t* pv = (uint8_t*)malloc(M);
        if (!mnf || !mxf || !pv) bad = 1;
#pragma omp for schedule(dynamic, 16)
        for (uint64_t k = 0; k < n_states; ++k) {
            if (bad) continue;
            const uint64_t s = states[k];
            uint8_t rn = reach_prev[s];
            uint32_t ct = ctl_prev[s];
            uint32_t st = step_prev[s];
            if (valid[s]) {
                const int is_cand = cand[s] != 0;
                const int already_reached = reach_prev[s] != 0;
                const int already_cert = ctl_prev[s] != 0xFFFFFFFFu;
                if (!((!is_cand && already_reached) || (is_cand && already_cert))) {
                    abstraction_row(c, &g, &u, s, mnf, mxf, pv);
                    uint32_t chosen;
                    if (state_step(&g, M, ps, pre_valid, pre_reach, mnf, mxf, pv, &chosen)) {
                        if (!already_reached) rn = 1;
                        if (!already_cert) {
                            ct = chosen;
                            if (!is_cand) st = iter;
                        }
                    }
                }
            }
            reach_next_out[k] = rn;
            ctl_out[k] = ct;
            step_out[k] = st;
        }
        free(mnf);
        free(mxf);
        free(pv);
    }
    free(pre_valid);
    free(pre_reach);
    return bad ? -3 : 0;
}
