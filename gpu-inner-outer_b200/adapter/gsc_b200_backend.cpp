// gsc_b200_backend.cpp -- the reference's CUDA backend entry points over libgsc_b200.
//
// The reference declares its GPU backend as two functions
// (include/gsc/cuda_api.hpp:87-88) and picks their implementation at link
// time (CMakeLists.txt:21-40): cuda/kernels.cu when CUDA is built,
// src/cuda_stubs.cpp otherwise.  This file is a third implementation of the
// same two functions.  It compiles against the reference's own headers
// (gsc/cuda_api.hpp and what it includes) plus include/gsc_b200.h, and links
// with libgsc_b200.so in place of kernels.cu.  The reference's CLI
// (src/main.cpp), tests (tests/test_small_case.cpp, tests/smoke_test.cpp) and
// result writer (src/result_io.cpp) build against it unchanged.
//
// run_case_cuda_u32 fills every GpuRunReport field that kernels.cu:492-875
// fills:
//   - result: masks, controller, reach_step, iteration count, stop message and
//     counts, copied from the device-resident solve (kernels.cu:776-836);
//   - state_grid / input_grid / budget / pair_count: the reference's own grid
//     builders and memory estimate, as prepare_case_gpu_minimal fills them
//     (abstraction.hpp:245-274, kernels.cu:505-511);
//   - kernel_timings / memory_stats / iteration_stats: the library's
//     per-phase CUDA-event timings (gsc_problem_phase_timings,
//     gsc_problem_iteration_timings).  Like kernels.cu, which synchronises
//     after every kernel to time it, the default solve runs the fixpoint from
//     the host loop with events around each phase (GSC_SOLVE_PROFILE).
//     Setting GSC_B200_SOLVE=graph runs it as one CUDA graph instead: faster,
//     and the per-kernel fields stay zero;
//   - abstraction_min_flat / max_flat / valid: the per-pair boxes in the
//     reference's layout, exported from the device as kernels.cu:785-824
//     copies them (GSC_B200_EXPORT_ABSTRACTION=0 skips them).
//
// Errors keep the reference's contract (kernels.cu:496-502, :856-858): no
// device leaves runtime_available false with "no CUDA device found"; any
// other failure leaves executed false with the reason in message.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gsc/cuda_api.hpp"
#include "gsc_b200.h"

namespace gsc {
namespace {

bool env_is(const char* name, const char* value) {
    const char* v = std::getenv(name);
    return v && std::strcmp(v, value) == 0;
}

gsc_model_desc model_of(const CaseConfig& cfg) {
    gsc_model_desc m{};
    for (int d = 0; d < kStateDim; ++d) {
        m.state_lb[d] = cfg.state_lb[d];
        m.state_ub[d] = cfg.state_ub[d];
        m.state_eta[d] = cfg.state_eta[d];
    }
    m.wrap_dim = cfg.wrap_dim;
    for (int d = 0; d < kInputDim; ++d) {
        m.input_lb[d] = cfg.input_lb[d];
        m.input_ub[d] = cfg.input_ub[d];
        m.input_eta[d] = cfg.input_eta[d];
    }
    m.sample_time = cfg.sample_time;
    m.integration_substeps = cfg.integration_substeps;
    return m;
}

// The query and the host arrays it points to (alive across the C calls).
struct Query {
    gsc_query_desc q{};
    std::vector<double> obstacles;
    std::vector<std::uint8_t> safe;
};

void fill_query(const CaseConfig& cfg, const Grid4D<std::uint32_t>& grid, Query* out) {
    gsc_query_desc& q = out->q;
    for (int d = 0; d < kStateDim; ++d) {
        q.disturbance_half_width[d] = cfg.disturbance_half_width[d];
        q.map_lb[d] = cfg.map.lb[d];
        q.map_ub[d] = cfg.map.ub[d];
    }
    for (const auto& o : cfg.obstacles) {
        out->obstacles.insert(out->obstacles.end(), o.lb, o.lb + kStateDim);
        out->obstacles.insert(out->obstacles.end(), o.ub, o.ub + kStateDim);
    }
    q.obstacle_count = static_cast<std::uint32_t>(cfg.obstacles.size());
    q.obstacles = out->obstacles.empty() ? nullptr : out->obstacles.data();
    switch (cfg.constraint_type) {
        case ConstraintType::kNone:
            q.constraint_kind = GSC_CONSTRAINT_NONE;
            break;
        case ConstraintType::kHyperbolic:
            q.constraint_kind = GSC_CONSTRAINT_HYPERBOLIC;
            q.constraint_params[0] = cfg.hyperbolic_params.a;
            q.constraint_params[1] = cfg.hyperbolic_params.b;
            q.constraint_params[2] = cfg.hyperbolic_params.c;
            break;
        case ConstraintType::kElliptic:
            q.constraint_kind = GSC_CONSTRAINT_ELLIPTIC;
            q.constraint_params[0] = cfg.elliptic_params.a;
            q.constraint_params[1] = cfg.elliptic_params.b;
            break;
        case ConstraintType::kCustom: {
            // A host predicate: evaluated at every cell centre with the
            // reference's own grid (grid.hpp:38-44), where the CPU method
            // evaluates it (config.cpp:119-123, abstraction.hpp:65-90).
            out->safe.assign(grid.total_size, 1);
            if (cfg.custom_constraint) {
                for (std::uint64_t s = 0; s < grid.total_size; ++s) {
                    double x[kStateDim];
                    grid.center(static_cast<std::uint32_t>(s), x);
                    out->safe[s] = cfg.custom_constraint(x) ? 1 : 0;
                }
            }
            q.constraint_kind = GSC_CONSTRAINT_NONE;
            q.safe_mask = out->safe.data();
            q.safe_mask_rank = 4;
            break;
        }
    }
    q.candidate_kind = GSC_CANDIDATE_RECT;
    for (int d = 0; d < kStateDim; ++d) {
        q.candidate[d] = cfg.candidate.lb[d];
        q.candidate[kStateDim + d] = cfg.candidate.ub[d];
    }
    q.max_iterations = cfg.max_iterations;
}

}  // namespace

bool cuda_backend_compiled() { return gsc_cuda_backend_compiled() != 0; }

GpuRunReport run_case_cuda_u32(const CaseConfig& cfg) {
    GpuRunReport report;
    report.compiled_with_cuda = true;
    report.state_grid = build_state_grid<std::uint32_t>(cfg.state_lb, cfg.state_ub, cfg.state_eta, cfg.wrap_dim);
    report.input_grid = build_input_grid(cfg.input_lb, cfg.input_ub, cfg.input_eta);
    report.budget = estimate_memory_budget(report.state_grid, report.input_grid);
    const std::uint64_t S = report.state_grid.total_size;
    const std::uint64_t M = report.input_grid.total_size;
    report.pair_count = S * M;

    gsc_context* ctx = nullptr;
    int st = gsc_context_create(0, nullptr, &ctx);
    if (st == GSC_ERR_NO_DEVICE) {
        report.message = "no CUDA device found";
        return report;
    }
    if (st != GSC_OK) {
        report.message = gsc_status_string(st);
        return report;
    }
    report.runtime_available = true;

    const gsc_model_desc model = model_of(cfg);
    Query query;
    fill_query(cfg, report.state_grid, &query);
    const bool graph = env_is("GSC_B200_SOLVE", "graph");
    const bool export_abs = !env_is("GSC_B200_EXPORT_ABSTRACTION", "0");

    gsc_abstraction* abs = nullptr;
    gsc_problem* prob = nullptr;
    auto& r = report.result;
    std::vector<std::uint64_t> new_reachable(static_cast<size_t>(cfg.max_iterations) + 1);
    std::vector<std::uint64_t> new_certified(new_reachable.size());
    gsc_result out{};
    const auto t0 = std::chrono::steady_clock::now();
    st = gsc_abstraction_create(ctx, &model, &abs);
    if (st == GSC_OK) st = gsc_problem_create(ctx, abs, &query.q, GSC_METHOD_AUTO, &prob);
    const auto t1 = std::chrono::steady_clock::now();
    if (st == GSC_OK) st = gsc_problem_solve(prob, graph ? GSC_SOLVE_GRAPH : GSC_SOLVE_PROFILE);
    const auto t2 = std::chrono::steady_clock::now();
    if (st == GSC_OK) {
        r.valid_mask.resize(S);
        r.candidate_mask.resize(S);
        r.reachable_mask.resize(S);
        r.controller.resize(S);
        r.reach_step.resize(S);
        out.valid_mask = r.valid_mask.data();
        out.candidate_mask = r.candidate_mask.data();
        out.reachable_mask = r.reachable_mask.data();
        out.controller = r.controller.data();
        out.reach_step = r.reach_step.data();
        out.iter_new_reachable = new_reachable.data();
        out.iter_new_certified = new_certified.data();
        out.iter_capacity = static_cast<std::uint32_t>(new_reachable.size());
        st = gsc_problem_read(prob, &out);
    }
    if (st == GSC_OK && export_abs) {
        report.abstraction_min_flat.resize(report.pair_count);
        report.abstraction_max_flat.resize(report.pair_count);
        report.abstraction_valid.resize(report.pair_count);
        st = gsc_problem_export_abstraction(prob, report.abstraction_min_flat.data(),
                                            report.abstraction_max_flat.data(), report.abstraction_valid.data());
    }
    if (st != GSC_OK) {
        report.message = std::string(gsc_status_string(st)) + ": " + gsc_last_error(ctx);
    } else {
        report.executed = true;
        r.iterations = out.iterations;
        r.converged = out.converged != 0;
        r.message = gsc_message_string(out.message);
        r.reachable_states = out.reachable_states;
        r.certified_candidate_states = out.certified_candidates;

        gsc_phase_timings ph{};
        gsc_problem_phase_timings(prob, &ph);
        auto& k = report.kernel_timings;
        k.abstraction_kernel_ms = ph.abstraction_kernel_ms;
        k.abstraction_memcpy_h2d_ms = ph.abstraction_memcpy_h2d_ms;
        k.scatter_mask_ms = ph.scatter_mask_ms;
        k.scan_axis0_ms = ph.scan_axis_ms[0];
        k.scan_axis1_ms = ph.scan_axis_ms[1];
        k.scan_axis2_ms = ph.scan_axis_ms[2];
        k.scan_axis3_ms = ph.scan_axis_ms[3];
        k.prefix_build_total_ms = ph.prefix_build_total_ms;
        k.pair_satisfaction_ms = ph.pair_satisfaction_ms;
        k.reduce_inputs_ms = ph.reduce_inputs_ms;
        k.iteration_memcpy_ms = ph.iteration_memcpy_ms;
        k.result_memcpy_d2h_ms = ph.result_memcpy_d2h_ms;
        k.total_kernel_ms = ph.total_kernel_ms;
        k.total_memcpy_ms = ph.total_memcpy_ms;
        k.total_compute_ms = ph.total_compute_ms;
        auto& m = report.memory_stats;
        m.total_allocated_bytes = ph.total_allocated_bytes;
        m.peak_usage_bytes = ph.peak_usage_bytes;
        m.abstraction_bytes = ph.abstraction_bytes;
        m.prefix_bytes = ph.prefix_bytes;
        m.iteration_bytes = ph.iteration_bytes;
        m.result_bytes = ph.result_bytes;

        // Wall-clock phases as kernels.cu:641 / :769 / :840 measure them.
        report.abstraction_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        report.solve_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
        report.total_ms = report.abstraction_ms + report.solve_ms;
        r.solve_ms = report.solve_ms;

        const std::uint32_t n = std::min<std::uint32_t>(out.iterations, out.iter_capacity);
        std::vector<double> it_ms(n), pre_ms(n), sat_ms(n), red_ms(n);
        gsc_problem_iteration_timings(prob, n, it_ms.data(), pre_ms.data(), sat_ms.data(), red_ms.data());
        const std::uint32_t timed = std::min<std::uint32_t>(n, ph.profiled_iterations);
        std::uint64_t reach = out.candidate_count, cert = 0;
        for (std::uint32_t i = 0; i < n; ++i) {
            IterationStats s;
            s.iteration = i + 1;
            s.newly_reachable = new_reachable[i];
            s.newly_certified = new_certified[i];
            reach += new_reachable[i];
            cert += new_certified[i];
            s.total_reachable = reach;
            s.total_certified = cert;
            if (i < timed) {
                s.iteration_ms = it_ms[i];
                s.prefix_build_ms = pre_ms[i];
                s.satisfaction_check_ms = sat_ms[i];
                s.reduction_ms = red_ms[i];
            }
            report.iteration_stats.push_back(s);
        }
    }
    gsc_problem_destroy(prob);
    gsc_abstraction_destroy(abs);
    gsc_context_destroy(ctx);
    return report;
}

}  // namespace gsc
