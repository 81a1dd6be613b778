// ref_gpu_driver.cpp -- runs the REFERENCE's own CUDA backend (BENCH INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile with nvcc for sm_100a against the reference's
// cuda/kernels.cu, headers and src/config.cpp where they lie; nothing of the
// reference is copied into this repository.  The binary lands in oracle/_ref/
// (git-ignored) and times run_case_cuda_u32 (cuda/kernels.cu:492-875) on the
// same GPU as this library, for the cases its backend can express (built-in
// constraint kinds, rectangular candidate sets).
//
//   gsc_ref_gpu <case.bin> <runs>   one JSON line per run: the reference's
//                                   abstraction, fixpoint and total times, its
//                                   kernel timings, and the result counts.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "gsc/cuda_api.hpp"
#include "ref_case.hpp"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: gsc_ref_gpu <case.bin> <runs>\n";
        return 1;
    }
    try {
        const orc_case c = ref_case::read_case(argv[1]);
        if (c.candidate_kind != ORC_CANDIDATE_RECT || c.constraint_kind > ORC_CONSTRAINT_ELLIPTIC) {
            std::cerr << "the reference's CUDA backend takes built-in constraints and rectangular candidates only\n";
            return 2;
        }
        gsc::CaseConfig cfg = ref_case::to_config(c);
        cfg.verbose = false;
        const int runs = std::atoi(argv[2]);
        for (int i = 0; i < runs; ++i) {
            const gsc::GpuRunReport r = gsc::run_case_cuda_u32(cfg);
            if (!r.executed) {
                std::cerr << "reference gpu run unavailable: " << r.message << '\n';
                return 2;
            }
            const auto& k = r.kernel_timings;
            std::printf(
                "{\"abstraction_ms\": %.4f, \"solve_ms\": %.4f, \"total_ms\": %.4f, \"iterations\": %u, "
                "\"reachable_states\": %llu, \"certified_candidates\": %llu, \"message\": \"%s\", "
                "\"pair_satisfaction_ms\": %.4f, \"prefix_build_ms\": %.4f, \"reduce_inputs_ms\": %.4f, "
                "\"iteration_memcpy_ms\": %.4f, \"result_memcpy_d2h_ms\": %.4f, \"device_bytes\": %llu}\n",
                r.abstraction_ms, r.solve_ms, r.total_ms, r.result.iterations,
                static_cast<unsigned long long>(r.result.reachable_states),
                static_cast<unsigned long long>(r.result.certified_candidate_states), r.result.message.c_str(),
                k.pair_satisfaction_ms, k.prefix_build_total_ms, k.reduce_inputs_ms, k.iteration_memcpy_ms,
                k.result_memcpy_d2h_ms, static_cast<unsigned long long>(r.memory_stats.total_allocated_bytes));
            std::fflush(stdout);
        }
        return 0;
    } catch (const std::exception& ex) {
        std::cerr << "error: " << ex.what() << '\n';
        return 1;
    }
}
