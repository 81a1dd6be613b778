// gsc/config.hpp -- the case description of the gsc API (host side of libgsc_b200).
//
// Field names and meanings follow the reference's CaseConfig
// (include/gsc/config.hpp:41-67) so that a .cfg file or a CaseConfig built in
// code means the same thing on both.  Two extensions carry the benchmark
// workloads, which the reference can only express through a custom predicate:
//   * ConstraintType::kQuadric: (x*x)*qa - (y*y)*qb <= c && fabs(y) <= ymax;
//   * CandidateShape::kEllipse: valid && (dx*dx)*wx + (dy*dy)*wy <= r2.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace gsc {

constexpr int kStateDim = 4;
constexpr int kInputDim = 2;

struct HyperRect4D {
    double lb[kStateDim]{};
    double ub[kStateDim]{};
};

enum class ConstraintType { kNone = 0, kHyperbolic = 1, kElliptic = 2, kQuadric = 3, kCustom = 4 };
enum class CandidateShape { kRect = 0, kEllipse = 1 };

struct HyperbolicConstraintParams {
    double a = 4.0;
    double b = 4.0;
    double c = 16.0;
};

struct EllipticConstraintParams {
    double a = 2.0;
    double b = 2.0;
};

struct QuadricConstraintParams {
    double qa = 1.0;
    double qb = 1.0;
    double c = 1.0;
    double ymax = 1.8;
};

struct EllipseCandidate {
    double cx = 0.0, cy = 0.0, wx = 1.0, wy = 1.0, r2 = 0.5;
};

using StateConstraintFn = std::function<bool(const double x[kStateDim])>;

struct CaseConfig {
    std::string name = "unicycle_default";
    double state_lb[kStateDim]{-2.0, -2.0, -3.141592653589793, 0.0};
    double state_ub[kStateDim]{2.0, 2.0, 3.141592653589793, 2.0};
    double state_eta[kStateDim]{0.5, 0.5, 0.7853981633974483, 0.5};
    int wrap_dim = 2;

    double input_lb[kInputDim]{-0.5, -1.0};
    double input_ub[kInputDim]{0.5, 1.0};
    double input_eta[kInputDim]{0.5, 1.0};

    HyperRect4D candidate{};
    CandidateShape candidate_shape = CandidateShape::kRect;
    EllipseCandidate candidate_ellipse{};
    HyperRect4D map{};
    std::vector<HyperRect4D> obstacles;

    ConstraintType constraint_type = ConstraintType::kNone;
    HyperbolicConstraintParams hyperbolic_params;
    EllipticConstraintParams elliptic_params;
    QuadricConstraintParams quadric_params;
    StateConstraintFn custom_constraint;   // evaluated on the host at cell centres

    double disturbance_half_width[kStateDim]{0.05, 0.05, 0.02, 0.02};
    double sample_time = 0.2;
    std::uint32_t integration_substeps = 32;
    std::uint32_t max_iterations = 32;
    bool verbose = true;
};

bool point_in_rect(const HyperRect4D& rect, const double x[kStateDim]);
bool satisfies_state_constraint(const CaseConfig& cfg, const double x[kStateDim]);

// The reference's built-in cases (config.cpp:129-241).
CaseConfig make_default_case();
CaseConfig make_wraparound_case();
CaseConfig make_smoke_case();
CaseConfig make_hyperbolic_case();
// The benchmark family: n = (nx, ny, ntheta, nv) states over x, y in [-2, 2],
// theta in [-pi, pi), v in [0, 1]; m = (m_a, m_omega) inputs.
CaseConfig make_unicycle_grid_case(const std::uint32_t n[4], const std::uint32_t m[2]);

// key = value parser with the reference's keys (config.cpp:243-347) plus
// quadric_* and candidate_shape / candidate_ellipse.  Throws on unknown keys.
CaseConfig load_case_config(const std::string& path);
CaseConfig parse_case_config(const std::string& text);

}  // namespace gsc
