// ref_driver.cpp -- runs the REFERENCE's own CPU method (TEST/BENCH INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile against the reference's headers and
// src/config.cpp where they lie (include/gsc/*.hpp, src/config.cpp of
// zzx-ur/gpu-inner-outer); nothing of the reference is copied into this
// repository.  The binary lands in oracle/_ref/ (git-ignored) and is used to
// (a) pin the C oracle against the reference and generate golden fixtures, and
// (b) time the reference CPU path as the bench's CPU baseline.
//
// Input: an orc_case struct (oracle/gsc_oracle.h) in a binary file.
//
//   gsc_ref full   <case.bin> <outdir>      prepare_case_cpu + solve_backward_cpu
//                                           (abstraction.hpp:276-307,
//                                           reachability.hpp:30-155), verbose,
//                                           outputs written as raw arrays.
//   gsc_ref sample <case.bin> <n_states> <seed> <threads>
//                                           times the reference's per-state
//                                           abstraction row (abstraction.hpp:168-208)
//                                           and the iteration-1 state body
//                                           (reachability.hpp:59-109) on a seeded
//                                           sample of states, split over threads.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "gsc/reachability.hpp"
#include "gsc_oracle.h"
#include "ref_case.hpp"

namespace {

using Clock = std::chrono::steady_clock;

using ref_case::read_case;
using ref_case::to_config;

void overwrite_candidate(const orc_case& c, gsc::PreparedCase<std::uint32_t>& p) {
    if (c.candidate_kind != ORC_CANDIDATE_ELLIPSE) return;
    for (std::uint64_t f = 0; f < p.state_grid.total_size; ++f) {
        double x[4];
        p.state_grid.center(static_cast<std::uint32_t>(f), x);
        const double dx = x[0] - c.cand[0];
        const double dy = x[1] - c.cand[1];
        const bool k = p.valid_mask[f] && ((dx * dx) * c.cand[2] + (dy * dy) * c.cand[3] <= c.cand[4]);
        p.candidate_mask[f] = k ? 1 : 0;
    }
}

template <typename T>
void dump(const std::string& path, const std::vector<T>& v) {
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

int run_full(const orc_case& c, const std::string& outdir) {
    const auto cfg = to_config(c);
    auto prepared = gsc::prepare_case_cpu<std::uint32_t>(cfg);
    overwrite_candidate(c, prepared);
    std::fflush(stdout);
    const auto result = gsc::solve_backward_cpu(prepared, cfg.max_iterations, true);
    std::fflush(stdout);
    dump(outdir + "/valid.u8", result.valid_mask);
    dump(outdir + "/candidate.u8", result.candidate_mask);
    dump(outdir + "/reachable.u8", result.reachable_mask);
    dump(outdir + "/controller.u32", result.controller);
    dump(outdir + "/reach_step.u32", result.reach_step);
    if (prepared.abstraction.pair_count <= (1ull << 26)) {
        dump(outdir + "/min_flat.u32", prepared.abstraction.min_flat);
        dump(outdir + "/max_flat.u32", prepared.abstraction.max_flat);
        dump(outdir + "/pair_valid.u8", prepared.abstraction.valid);
    }
    std::uint64_t valid_pairs = 0;
    for (auto v : prepared.abstraction.valid) valid_pairs += v;
    std::printf("SUMMARY states=%llu inputs=%llu iterations=%u converged=%d reachable=%llu certified=%llu "
                "valid_pairs=%llu abstraction_ms=%.3f solve_ms=%.3f\n",
                static_cast<unsigned long long>(prepared.state_grid.total_size),
                static_cast<unsigned long long>(prepared.input_grid.total_size), result.iterations,
                result.converged ? 1 : 0, static_cast<unsigned long long>(result.reachable_states),
                static_cast<unsigned long long>(result.certified_candidate_states),
                static_cast<unsigned long long>(valid_pairs), prepared.abstraction_ms, result.solve_ms);
    std::printf("MESSAGE %s\n", result.message.c_str());
    return 0;
}

// The reference's per-state abstraction row (abstraction.hpp:168-208) and
// iteration body (reachability.hpp:59-109), timed on a sample of states.
int run_sample(const orc_case& c, std::uint64_t n, std::uint64_t seed, unsigned threads) {
    const auto cfg = to_config(c);
    const auto grid = gsc::build_state_grid<std::uint32_t>(cfg.state_lb, cfg.state_ub, cfg.state_eta, cfg.wrap_dim);
    const auto igrid = gsc::build_input_grid(cfg.input_lb, cfg.input_ub, cfg.input_eta);
    gsc::Unicycle4DModel model;
    model.sample_time = cfg.sample_time;
    model.integration_substeps = cfg.integration_substeps;
    for (int d = 0; d < 4; ++d) model.disturbance_half_width[d] = cfg.disturbance_half_width[d];
    const auto valid = gsc::build_valid_mask(grid, cfg);
    auto cand = gsc::build_candidate_mask(grid, cfg.candidate);
    if (c.candidate_kind == ORC_CANDIDATE_ELLIPSE) {
        for (std::uint64_t f = 0; f < grid.total_size; ++f) {
            double x[4];
            grid.center(static_cast<std::uint32_t>(f), x);
            const double dx = x[0] - c.cand[0], dy = x[1] - c.cand[1];
            cand[f] = (valid[f] && ((dx * dx) * c.cand[2] + (dy * dy) * c.cand[3] <= c.cand[4])) ? 1 : 0;
        }
    }
    const auto t_pre0 = Clock::now();
    const auto prefix_valid = gsc::build_prefix_sum_cpu(grid, valid);
    const auto prefix_reach = gsc::build_prefix_sum_cpu(grid, cand);
    const auto t_pre1 = Clock::now();
    const double prefix_ms = std::chrono::duration<double, std::milli>(t_pre1 - t_pre0).count() / 2.0;

    // The sample is made of contiguous runs of states (as the reference's own
    // loop visits them, so its caches see the same access pattern), one run
    // per thread, each starting at a seeded offset.
    std::mt19937_64 rng(seed);
    std::vector<std::uint64_t> states;
    states.reserve(n);
    const std::uint64_t run = std::max<std::uint64_t>(1, n / threads);
    while (states.size() < n) {
        const std::uint64_t len = std::min<std::uint64_t>(run, n - states.size());
        const std::uint64_t start = rng() % (grid.total_size - std::min<std::uint64_t>(len, grid.total_size) + 1);
        for (std::uint64_t k = 0; k < len && start + k < grid.total_size; ++k) states.push_back(start + k);
        if (len == 0) break;
    }
    n = states.size();
    const std::uint64_t M = igrid.total_size;

    std::vector<std::uint32_t> mnf(n * M), mxf(n * M);
    std::vector<std::uint8_t> pv(n * M);
    auto range_of = [&](unsigned t, std::uint64_t* b, std::uint64_t* e) {
        *b = n * t / threads;
        *e = n * (t + 1) / threads;
    };
    auto worker_abs = [&](unsigned t) {
        std::uint64_t kb, ke;
        range_of(t, &kb, &ke);
        for (std::uint64_t k = kb; k < ke; ++k) {
            const std::uint64_t state = states[k];
            double x[4];
            grid.center(static_cast<std::uint32_t>(state), x);
            if (cfg.constraint_type != gsc::ConstraintType::kNone && !gsc::satisfies_state_constraint(cfg, x)) continue;
            for (std::uint64_t input = 0; input < M; ++input) {
                double u[2], mn[4], mx[4];
                igrid.center(static_cast<gsc::InputIndex>(input), u);
                model.successor_box(x, u, grid.eta, mn, mx);
                gsc::IndexBox4D box{};
                if (!gsc::continuous_box_to_index_box(grid, mn, mx, &box)) continue;
                if (!gsc::box_satisfies_constraint(grid, box, cfg)) continue;
                mnf[k * M + input] = grid.flatten(box.min);
                mxf[k * M + input] = grid.flatten(box.max);
                pv[k * M + input] = 1;
            }
        }
    };
    std::atomic<std::uint64_t> hits{0};
    auto worker_fix = [&](unsigned t) {
        std::uint64_t local = 0;
        std::uint64_t kb, ke;
        range_of(t, &kb, &ke);
        for (std::uint64_t k = kb; k < ke; ++k) {
            const std::uint64_t state = states[k];
            if (!valid[state]) continue;
            for (std::uint64_t input = 0; input < M; ++input) {
                const std::uint64_t pair = k * M + input;
                if (!pv[pair]) continue;
                const auto vc = gsc::query_box_count(grid, prefix_valid, mnf[pair], mxf[pair]);
                if (vc == 0) continue;
                const auto rc = gsc::query_box_count(grid, prefix_reach, mnf[pair], mxf[pair]);
                if (rc == vc) {
                    ++local;
                    break;
                }
            }
        }
        hits += local;
    };
    auto run_threads = [&](auto&& fn) {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < threads; ++t) pool.emplace_back(fn, t);
        for (auto& th : pool) th.join();
    };
    const auto a0 = Clock::now();
    run_threads(worker_abs);
    const auto a1 = Clock::now();
    run_threads(worker_fix);
    const auto a2 = Clock::now();
    const double abs_ms = std::chrono::duration<double, std::milli>(a1 - a0).count();
    const double fix_ms = std::chrono::duration<double, std::milli>(a2 - a1).count();
    std::printf("SAMPLE states=%llu grid_states=%llu inputs=%llu threads=%u abstraction_ms=%.3f iteration_ms=%.3f "
                "prefix_ms=%.3f satisfied=%llu\n",
                static_cast<unsigned long long>(n), static_cast<unsigned long long>(grid.total_size),
                static_cast<unsigned long long>(M), threads, abs_ms, fix_ms, prefix_ms,
                static_cast<unsigned long long>(hits.load()));
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc >= 4 && std::strcmp(argv[1], "full") == 0) return run_full(read_case(argv[2]), argv[3]);
        if (argc >= 6 && std::strcmp(argv[1], "sample") == 0)
            return run_sample(read_case(argv[2]), std::stoull(argv[3]), std::stoull(argv[4]),
                              static_cast<unsigned>(std::stoul(argv[5])));
        std::fprintf(stderr, "usage: gsc_ref full <case.bin> <outdir> | sample <case.bin> <n> <seed> <threads>\n");
        return 1;
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "error: %s\n", ex.what());
        return 1;
    }
}
