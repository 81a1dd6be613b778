// cuda_api.cpp -- run_case_cuda_u32 (the reference's backend call,
// cuda/kernels.cu:492-875) implemented over libgsc_b200's C ABI.
#include "gsc/cuda_api.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <stdexcept>

#include "gsc_b200.h"

namespace gsc {

namespace {

gsc_model_desc model_of(const CaseConfig& cfg) {
    gsc_model_desc m{};
    for (int d = 0; d < 4; ++d) {
        m.state_lb[d] = cfg.state_lb[d];
        m.state_ub[d] = cfg.state_ub[d];
        m.state_eta[d] = cfg.state_eta[d];
    }
    m.wrap_dim = cfg.wrap_dim;
    for (int d = 0; d < 2; ++d) {
        m.input_lb[d] = cfg.input_lb[d];
        m.input_ub[d] = cfg.input_ub[d];
        m.input_eta[d] = cfg.input_eta[d];
    }
    m.sample_time = cfg.sample_time;
    m.integration_substeps = cfg.integration_substeps;
    return m;
}

// Everything the query points to must outlive the C calls.
struct QueryStorage {
    gsc_query_desc q{};
    std::vector<double> obstacles;
    std::vector<std::uint8_t> safe;
};

void query_of(const CaseConfig& cfg, const std::uint32_t shape[4], QueryStorage* qs) {
    gsc_query_desc& q = qs->q;
    for (int d = 0; d < 4; ++d) {
        q.disturbance_half_width[d] = cfg.disturbance_half_width[d];
        q.map_lb[d] = cfg.map.lb[d];
        q.map_ub[d] = cfg.map.ub[d];
    }
    for (const auto& o : cfg.obstacles) {
        qs->obstacles.insert(qs->obstacles.end(), o.lb, o.lb + 4);
        qs->obstacles.insert(qs->obstacles.end(), o.ub, o.ub + 4);
    }
    q.obstacle_count = static_cast<std::uint32_t>(cfg.obstacles.size());
    q.obstacles = qs->obstacles.empty() ? nullptr : qs->obstacles.data();
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
        case ConstraintType::kQuadric:
            q.constraint_kind = GSC_CONSTRAINT_QUADRIC;
            q.constraint_params[0] = cfg.quadric_params.qa;
            q.constraint_params[1] = cfg.quadric_params.qb;
            q.constraint_params[2] = cfg.quadric_params.c;
            q.constraint_params[3] = cfg.quadric_params.ymax;
            break;
        case ConstraintType::kCustom: {
            // The predicate is host code: evaluate it at every cell centre
            // (grid.hpp:38-44), exactly where the reference evaluates it.
            const std::uint64_t S = std::uint64_t(shape[0]) * shape[1] * shape[2] * shape[3];
            qs->safe.assign(S, 1);
            if (cfg.custom_constraint) {
                std::uint32_t idx[4];
                for (std::uint64_t s = 0; s < S; ++s) {
                    std::uint64_t r = s;
                    for (int d = 0; d < 4; ++d) {
                        idx[d] = static_cast<std::uint32_t>(r % shape[d]);
                        r /= shape[d];
                    }
                    double x[4];
                    for (int d = 0; d < 4; ++d)
                        x[d] = cfg.state_lb[d] + (static_cast<double>(idx[d]) + 0.5) * cfg.state_eta[d];
                    qs->safe[s] = cfg.custom_constraint(x) ? 1 : 0;
                }
            }
            q.constraint_kind = GSC_CONSTRAINT_NONE;
            q.safe_mask = qs->safe.data();
            q.safe_mask_rank = 4;
            break;
        }
    }
    if (cfg.candidate_shape == CandidateShape::kRect) {
        q.candidate_kind = GSC_CANDIDATE_RECT;
        for (int d = 0; d < 4; ++d) {
            q.candidate[d] = cfg.candidate.lb[d];
            q.candidate[4 + d] = cfg.candidate.ub[d];
        }
    } else {
        q.candidate_kind = GSC_CANDIDATE_ELLIPSE;
        const EllipseCandidate& e = cfg.candidate_ellipse;
        q.candidate[0] = e.cx;
        q.candidate[1] = e.cy;
        q.candidate[2] = e.wx;
        q.candidate[3] = e.wy;
        q.candidate[4] = e.r2;
    }
    q.max_iterations = cfg.max_iterations;
}

// estimate_memory_budget (abstraction.hpp:211-243): the reference's byte
// counts for its own device layout (u32 flats, u8 masks, u64 prefix tables).
MemoryBudget reference_budget(const GridShape& sg, const GridShape& ig) {
    const std::uint64_t S = sg.total_size, P = S * ig.total_size;
    std::uint64_t T = 1;
    for (int d = 0; d < kStateDim; ++d) T *= static_cast<std::uint64_t>(sg.shape[d]) + 1;
    MemoryBudget b;
    b.pair_min_bytes = P * 4;
    b.pair_max_bytes = P * 4;
    b.pair_valid_bytes = P;
    b.pair_satisfied_bytes = P;
    b.reachable_prev_bytes = S;
    b.reachable_next_bytes = S;
    b.valid_mask_bytes = S;
    b.candidate_mask_bytes = S;
    b.controller_bytes = S * 4;
    b.reach_step_bytes = S * 4;
    b.prefix_reachable_bytes = T * 8;
    b.prefix_valid_bytes = T * 8;
    b.total_bytes = b.pair_min_bytes + b.pair_max_bytes + b.pair_valid_bytes + b.pair_satisfied_bytes +
                    b.reachable_prev_bytes + b.reachable_next_bytes + b.valid_mask_bytes + b.candidate_mask_bytes +
                    b.controller_bytes + b.reach_step_bytes + b.prefix_reachable_bytes + b.prefix_valid_bytes;
    return b;
}

}  // namespace

bool cuda_backend_compiled() { return gsc_cuda_backend_compiled() != 0; }

GpuRunReport run_case_cuda_u32(const CaseConfig& cfg) { return run_case_cuda_u32(cfg, RunOptions{}); }

GpuRunReport run_case_cuda_u32(const CaseConfig& cfg, const RunOptions& opt) {
    GpuRunReport report;
    report.compiled_with_cuda = true;
    const gsc_model_desc m = model_of(cfg);
    std::uint32_t shape[4], ishape[2];
    int st = gsc_grid_shape(&m, shape, ishape);
    if (st != GSC_OK) {
        report.message = gsc_status_string(st);
        return report;
    }
    std::uint64_t S = 1;
    for (int d = 0; d < 4; ++d) {
        report.state_grid.shape[d] = shape[d];
        S *= shape[d];
    }
    report.state_grid.total_size = S;
    report.input_grid.shape[0] = ishape[0];
    report.input_grid.shape[1] = ishape[1];
    report.input_grid.total_size = std::uint64_t(ishape[0]) * ishape[1];
    report.pair_count = S * report.input_grid.total_size;

    gsc_context* ctx = nullptr;
    st = gsc_context_create(opt.device, nullptr, &ctx);
    if (st == GSC_ERR_NO_DEVICE) {   // kernels.cu:497-502
        report.message = "no CUDA device found";
        return report;
    }
    if (st != GSC_OK) {
        report.message = gsc_status_string(st);
        return report;
    }
    report.runtime_available = true;
    QueryStorage qs;
    query_of(cfg, shape, &qs);
    gsc_abstraction* abs = nullptr;
    gsc_problem* p = nullptr;
    auto& r = report.result;
    std::vector<std::uint64_t> nr(static_cast<size_t>(cfg.max_iterations) + 1), nc(nr.size());
    gsc_result out{};
    gsc_timings t{};
    const auto t0 = std::chrono::steady_clock::now();
    st = gsc_abstraction_create(ctx, &m, &abs);
    if (st == GSC_OK) st = gsc_problem_create(ctx, abs, &qs.q, opt.method, &p);
    const std::uint32_t solve_flags = opt.profile ? GSC_SOLVE_PROFILE : opt.graph ? GSC_SOLVE_GRAPH : 0;
    if (st == GSC_OK) st = gsc_problem_solve(p, solve_flags);
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
        out.iter_new_reachable = nr.data();
        out.iter_new_certified = nc.data();
        out.iter_capacity = static_cast<std::uint32_t>(nr.size());
        st = gsc_problem_read(p, &out);
    }
    if (st == GSC_OK && opt.export_abstraction) {
        report.abstraction_min_flat.resize(report.pair_count);
        report.abstraction_max_flat.resize(report.pair_count);
        report.abstraction_valid.resize(report.pair_count);
        st = gsc_problem_export_abstraction(p, report.abstraction_min_flat.data(), report.abstraction_max_flat.data(),
                                            report.abstraction_valid.data());
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (st != GSC_OK) {   // kernels.cu:856-858: the error becomes the report's message
        report.message = std::string(gsc_status_string(st)) + ": " + gsc_last_error(ctx);
    } else {
        gsc_problem_timings(p, &t);
        report.executed = true;
        r.iterations = out.iterations;
        r.converged = out.converged != 0;
        r.message = gsc_message_string(out.message);
        r.reachable_states = out.reachable_states;
        r.certified_candidate_states = out.certified_candidates;
        r.solve_ms = report.solve_ms = t.solve_ms;
        gsc_phase_timings ph{};
        gsc_problem_phase_timings(p, &ph);
        KernelTimings& k = report.kernel_timings;
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
        k.prepare_ms = t.prepare_ms;
        k.solve_ms = t.solve_ms;
        GpuMemoryStats& ms = report.memory_stats;
        ms.total_allocated_bytes = ph.total_allocated_bytes;
        ms.peak_usage_bytes = ph.peak_usage_bytes;
        ms.abstraction_bytes = ph.abstraction_bytes;
        ms.prefix_bytes = ph.prefix_bytes;
        ms.iteration_bytes = ph.iteration_bytes;
        ms.result_bytes = ph.result_bytes;
        report.budget = reference_budget(report.state_grid, report.input_grid);
        report.abstraction_ms = t.abstraction_ms + t.prepare_ms;
        report.total_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        const std::uint32_t n = std::min<std::uint32_t>(out.iterations, out.iter_capacity);
        std::vector<double> it_ms(n), pre_ms(n), sat_ms(n), red_ms(n);
        gsc_problem_iteration_timings(p, n, it_ms.data(), pre_ms.data(), sat_ms.data(), red_ms.data());
        const std::uint32_t timed = opt.profile ? std::min<std::uint32_t>(n, ph.profiled_iterations) : 0;
        std::uint64_t reach = out.candidate_count, cert = 0;
        for (std::uint32_t i = 0; i < n; ++i) {
            IterationStats s;
            s.iteration = i + 1;
            s.newly_reachable = nr[i];
            s.newly_certified = nc[i];
            reach += nr[i];
            cert += nc[i];
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
    gsc_problem_destroy(p);
    gsc_abstraction_destroy(abs);
    gsc_context_destroy(ctx);
    return report;
}

}  // namespace gsc
