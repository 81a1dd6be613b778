// ref_case.hpp -- the oracle's case description (oracle/gsc_oracle.h) as a
// reference CaseConfig, for the drivers of the reference's own code
// (TEST/BENCH INFRASTRUCTURE ONLY; compiled against the reference's headers
// where they lie).
#pragma once

#include <cmath>
#include <fstream>
#include <stdexcept>

#include "gsc/config.hpp"
#include "gsc_oracle.h"

namespace ref_case {

inline orc_case read_case(const char* path) {
    orc_case c;
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open case file");
    in.read(reinterpret_cast<char*>(&c), sizeof(c));
    if (in.gcount() != static_cast<std::streamsize>(sizeof(c))) throw std::runtime_error("short case file");
    return c;
}

// Build a reference CaseConfig from the oracle's case description.  The
// quadric safe set becomes ConstraintType::kCustom with the same expression.
inline gsc::CaseConfig to_config(const orc_case& c) {
    gsc::CaseConfig cfg;
    cfg.name = "oracle_case";
    for (int d = 0; d < 4; ++d) {
        cfg.state_lb[d] = c.state_lb[d];
        cfg.state_ub[d] = c.state_ub[d];
        cfg.state_eta[d] = c.state_eta[d];
        cfg.disturbance_half_width[d] = c.dhw[d];
        cfg.map.lb[d] = c.map_lb[d];
        cfg.map.ub[d] = c.map_ub[d];
    }
    cfg.wrap_dim = c.wrap_dim;
    for (int d = 0; d < 2; ++d) {
        cfg.input_lb[d] = c.input_lb[d];
        cfg.input_ub[d] = c.input_ub[d];
        cfg.input_eta[d] = c.input_eta[d];
    }
    cfg.sample_time = c.sample_time;
    cfg.integration_substeps = c.substeps;
    cfg.max_iterations = c.max_iterations;
    cfg.obstacles.clear();
    for (int o = 0; o < c.n_obstacles; ++o) {
        gsc::HyperRect4D r;
        for (int d = 0; d < 4; ++d) {
            r.lb[d] = c.obstacles[o][d];
            r.ub[d] = c.obstacles[o][4 + d];
        }
        cfg.obstacles.push_back(r);
    }
    switch (c.constraint_kind) {
        case ORC_CONSTRAINT_NONE:
            cfg.constraint_type = gsc::ConstraintType::kNone;
            break;
        case ORC_CONSTRAINT_HYPERBOLIC:
            cfg.constraint_type = gsc::ConstraintType::kHyperbolic;
            cfg.hyperbolic_params.a = c.cparam[0];
            cfg.hyperbolic_params.b = c.cparam[1];
            cfg.hyperbolic_params.c = c.cparam[2];
            break;
        case ORC_CONSTRAINT_ELLIPTIC:
            cfg.constraint_type = gsc::ConstraintType::kElliptic;
            cfg.elliptic_params.a = c.cparam[0];
            cfg.elliptic_params.b = c.cparam[1];
            break;
        default: {
            cfg.constraint_type = gsc::ConstraintType::kCustom;
            const double qa = c.cparam[0], qb = c.cparam[1], cc = c.cparam[2], ymax = c.cparam[3];
            cfg.custom_constraint = [qa, qb, cc, ymax](const double x[gsc::kStateDim]) {
                return ((x[0] * x[0]) * qa - (x[1] * x[1]) * qb <= cc) && (std::fabs(x[1]) <= ymax);
            };
        }
    }
    if (c.candidate_kind == ORC_CANDIDATE_RECT) {
        for (int d = 0; d < 4; ++d) {
            cfg.candidate.lb[d] = c.cand[d];
            cfg.candidate.ub[d] = c.cand[4 + d];
        }
    } else {
        // An empty rectangle; the ellipse mask is written after preparation.
        for (int d = 0; d < 4; ++d) {
            cfg.candidate.lb[d] = 1.0;
            cfg.candidate.ub[d] = -1.0;
        }
    }
    cfg.verbose = true;
    return cfg;
}

}  // namespace ref_case
