/*
 * gsc_oracle.h -- CPU oracle for the grid symbolic-control hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * CPU method (zzx-ur/gpu-inner-outer, namespace gsc).  Only the tests, the
 * smoke entry point and the bench's CPU-baseline leg may load it, and only as
 * the checker.  The product library never links, loads or calls it.
 *
 * Parity pin: the restatement is checked against (1) the reference's own CPU
 * code compiled from its sources into oracle/_ref (see oracle/Makefile and
 * oracle/ref_driver.cpp), and (2) the published demo run of the reference
 * (README.md:44-98: reachable 1,142,689, 12 iterations, per-iteration counts).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef GSC_ORACLE_H
#define GSC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_OBSTACLES 16

/* Constraint kinds.  0..2 follow include/gsc/config.hpp:19-24
 * (ConstraintType::kNone/kHyperbolic/kElliptic).  3 is the quadric safe set
 * used by the benchmark configurations ((x*x)*qa - (y*y)*qb <= c and
 * fabs(y) <= ymax); the reference expresses it as ConstraintType::kCustom
 * with a predicate of exactly that expression (config.cpp:119-123). */
enum { ORC_CONSTRAINT_NONE = 0, ORC_CONSTRAINT_HYPERBOLIC = 1,
       ORC_CONSTRAINT_ELLIPTIC = 2, ORC_CONSTRAINT_QUADRIC = 3 };

/* Candidate kinds.  0 = inclusive hyper-rectangle (abstraction.hpp:65-75,
 * point_in_rect config.cpp:80-87).  1 = ellipse in (x, y) intersected with
 * the valid mask: valid && (dx*dx)*wx + (dy*dy)*wy <= r2, dx = x - cx,
 * dy = y - cy (the benchmark configurations' candidate set). */
enum { ORC_CANDIDATE_RECT = 0, ORC_CANDIDATE_ELLIPSE = 1 };

enum { ORC_MSG_NONE = 0, ORC_MSG_CONVERGED = 1, ORC_MSG_STALLED = 2,
       ORC_MSG_MAX_ITER = 3 };

typedef struct {
    double state_lb[4], state_ub[4], state_eta[4];
    int32_t wrap_dim;
    double input_lb[2], input_ub[2], input_eta[2];
    double sample_time;
    uint32_t substeps;
    double dhw[4];                 /* disturbance_half_width */
    int32_t constraint_kind;
    double cparam[4];              /* hyperbolic a,b,c | elliptic a,b | quadric qa,qb,c,ymax */
    double map_lb[4], map_ub[4];
    int32_t n_obstacles;
    double obstacles[ORC_MAX_OBSTACLES][8];   /* lb[4], ub[4] */
    int32_t candidate_kind;
    double cand[8];                /* rect: lb[4], ub[4]; ellipse: cx, cy, wx, wy, r2 */
    uint32_t max_iterations;
} orc_case;

typedef struct {
    uint32_t shape[4];
    uint32_t input_shape[2];
    uint64_t states;
    uint64_t inputs;
    uint64_t pairs;
    uint32_t iterations;
    int32_t converged;
    int32_t message;               /* ORC_MSG_* */
    uint64_t reachable_states;
    uint64_t certified_candidates;
    uint64_t candidate_count;
    uint64_t valid_count;
    uint64_t valid_pairs;          /* abstraction pairs with valid = 1 */
    double abstraction_ms;
    double solve_ms;
} orc_summary;

/* Grid shapes exactly as build_state_grid / build_input_grid (grid.hpp:103-168).
 * Returns 0 on success, -1 on a rejected configuration. */
int orc_shapes(const orc_case* c, uint32_t shape[4], uint32_t input_shape[2]);

/* Valid / candidate masks (abstraction.hpp:65-106, with the ellipse candidate
 * extension).  Returns -1 if the candidate set contains an invalid state
 * (abstraction.hpp:291-295). */
int orc_masks(const orc_case* c, uint8_t* valid, uint8_t* candidate);

/* Per-pair abstraction (abstraction.hpp:161-209): pair = state * M + input. */
int orc_abstraction(const orc_case* c, uint32_t* min_flat, uint32_t* max_flat,
                    uint8_t* pair_valid, int nthreads);

/* 4-D inclusive prefix sum with a zero first plane per dimension
 * (prefix_sum.hpp:15-63, layout grid.hpp:253-269).  out has prod(shape+1). */
void orc_prefix(const uint32_t shape[4], const uint8_t* mask, uint64_t* out);

/* Box count of a (min_flat, max_flat) pair (prefix_sum.hpp:65-105). */
uint64_t orc_query(const uint32_t shape[4], int wrap_dim, const uint64_t* prefix,
                   uint32_t min_flat, uint32_t max_flat);

/* Full CPU method: masks, abstraction, backward fixpoint
 * (abstraction.hpp:276-307 then reachability.hpp:30-155).  Any output pointer
 * may be NULL.  iter_new_reach / iter_new_cert hold iter_cap entries. */
int orc_solve(const orc_case* c, uint8_t* valid, uint8_t* candidate,
              uint8_t* reachable, uint32_t* controller, uint32_t* reach_step,
              uint64_t* iter_new_reach, uint64_t* iter_new_cert, uint32_t iter_cap,
              orc_summary* out, int nthreads);

/* Spot oracle: recompute one fixpoint iteration for a list of states, given
 * the previous iteration's reachable mask and controller (the Jacobi update
 * of reachability.hpp:53-109 is a pure function of these).  For each listed
 * state it writes reachable_next, controller and reach_step after iteration
 * `iter`.  valid/candidate are the full masks. */
int orc_spot_step(const orc_case* c, const uint8_t* valid, const uint8_t* candidate,
                  const uint8_t* reach_prev, const uint32_t* controller_prev,
                  const uint32_t* reach_step_prev, uint32_t iter,
                  const uint64_t* states, uint64_t n_states,
                  uint8_t* reach_next_out, uint32_t* controller_out,
                  uint32_t* reach_step_out, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
