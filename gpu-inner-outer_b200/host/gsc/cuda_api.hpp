// gsc/cuda_api.hpp -- the reference's backend entry points, over libgsc_b200's C ABI.
//
// Same names and report fields as include/gsc/cuda_api.hpp:11-88 of the
// reference, so code written against run_case_cuda_u32 keeps working.  The
// abstraction arrays of the report are filled only when requested (they are
// P-sized; keeping them on the device is the point of the B200 design).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "gsc/config.hpp"

namespace gsc {

using InputIndex = std::uint32_t;
using ReachStep = std::uint32_t;
constexpr InputIndex kInvalidInput = 0xFFFFFFFFu;
constexpr ReachStep kUnreachableStep = 0xFFFFFFFFu;

struct SolveResult {
    std::vector<std::uint8_t> valid_mask;
    std::vector<std::uint8_t> candidate_mask;
    std::vector<std::uint8_t> reachable_mask;
    std::vector<InputIndex> controller;
    std::vector<ReachStep> reach_step;
    std::uint32_t iterations = 0;
    bool converged = false;
    std::string message;
    std::uint64_t reachable_states = 0;
    std::uint64_t certified_candidate_states = 0;
    double solve_ms = 0.0;
};

struct IterationStats {
    std::uint32_t iteration = 0;
    std::uint64_t newly_reachable = 0;
    std::uint64_t newly_certified = 0;
    std::uint64_t total_reachable = 0;
    std::uint64_t total_certified = 0;
    double iteration_ms = 0.0;            // profiled solves only (RunOptions::profile)
    double prefix_build_ms = 0.0;
    double satisfaction_check_ms = 0.0;
    double reduction_ms = 0.0;
};

// Every field of the reference's KernelTimings (cuda_api.hpp:24-48), filled
// from gsc_problem_phase_timings.  The per-kernel fields need a profiled solve
// (RunOptions::profile); prepare_ms and solve_ms are this mirror's own.
struct KernelTimings {
    double abstraction_kernel_ms = 0.0;
    double abstraction_memcpy_h2d_ms = 0.0;
    double scatter_mask_ms = 0.0;
    double scan_axis0_ms = 0.0;
    double scan_axis1_ms = 0.0;
    double scan_axis2_ms = 0.0;
    double scan_axis3_ms = 0.0;
    double prefix_build_total_ms = 0.0;
    double pair_satisfaction_ms = 0.0;
    double reduce_inputs_ms = 0.0;
    double iteration_memcpy_ms = 0.0;
    double result_memcpy_d2h_ms = 0.0;
    double total_kernel_ms = 0.0;
    double total_memcpy_ms = 0.0;
    double total_compute_ms = 0.0;
    double prepare_ms = 0.0;              // masks and quantised boxes
    double solve_ms = 0.0;                // the device fixpoint
};

// The reference's GpuMemoryStats (cuda_api.hpp:51-58).
struct GpuMemoryStats {
    std::uint64_t total_allocated_bytes = 0;
    std::uint64_t peak_usage_bytes = 0;
    std::uint64_t abstraction_bytes = 0;
    std::uint64_t prefix_bytes = 0;
    std::uint64_t iteration_bytes = 0;
    std::uint64_t result_bytes = 0;
};

// The reference's MemoryBudget (abstraction.hpp:16-30): its planning
// estimate for the reference's own device layout (estimate_memory_budget,
// abstraction.hpp:211-243), which run_case_cuda_u32 reports as `budget`.
struct MemoryBudget {
    std::uint64_t pair_min_bytes = 0;
    std::uint64_t pair_max_bytes = 0;
    std::uint64_t pair_valid_bytes = 0;
    std::uint64_t pair_satisfied_bytes = 0;
    std::uint64_t reachable_prev_bytes = 0;
    std::uint64_t reachable_next_bytes = 0;
    std::uint64_t valid_mask_bytes = 0;
    std::uint64_t candidate_mask_bytes = 0;
    std::uint64_t controller_bytes = 0;
    std::uint64_t reach_step_bytes = 0;
    std::uint64_t prefix_reachable_bytes = 0;
    std::uint64_t prefix_valid_bytes = 0;
    std::uint64_t total_bytes = 0;
};

struct GridShape {
    std::uint32_t shape[kStateDim]{};
    std::uint64_t total_size = 0;
};

struct GpuRunReport {
    bool compiled_with_cuda = false;
    bool runtime_available = false;
    bool executed = false;
    std::string message;
    double abstraction_ms = 0.0;
    double solve_ms = 0.0;
    double total_ms = 0.0;
    SolveResult result;
    GridShape state_grid;
    GridShape input_grid;
    MemoryBudget budget;
    std::uint64_t pair_count = 0;
    std::vector<IterationStats> iteration_stats;
    KernelTimings kernel_timings;
    GpuMemoryStats memory_stats;
    std::vector<std::uint32_t> abstraction_min_flat;
    std::vector<std::uint32_t> abstraction_max_flat;
    std::vector<std::uint8_t> abstraction_valid;
};

struct RunOptions {
    int device = 0;
    std::uint32_t method = 0;          // GSC_METHOD_*
    bool graph = true;                 // one CUDA graph for the whole fixpoint
    bool export_abstraction = false;   // fill abstraction_* (P-sized host copies)
    bool profile = false;              // host-loop solve with per-phase events (fills the per-kernel
                                       // KernelTimings and IterationStats times; overrides graph)
};

bool cuda_backend_compiled();
GpuRunReport run_case_cuda_u32(const CaseConfig& cfg);
GpuRunReport run_case_cuda_u32(const CaseConfig& cfg, const RunOptions& options);

}  // namespace gsc
