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
//   gsc_ref bench <case.bin> <threads> <warmup> <steps> <single>
//                                           builds the whole abstraction once
//                                           (rows split over threads, untimed),
//                                           then times warmup + steps full-grid
//                                           fixpoint iterations from the start
//                                           state: the reachable prefix build
//                                           (prefix_sum.hpp:15-63) and every
//                                           state's body (reachability.hpp:53-109),
//                                           states split over threads.  With
//                                           single=1 it also times one iteration
//                                           of solve_backward_cpu itself, as
//                                           shipped (one thread).
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

// The whole abstraction of a case with the reference's own per-pair steps
// (abstraction.hpp:161-209, the loop of build_abstraction_cpu), its states
// split over threads.
gsc::PreparedCase<std::uint32_t> prepare_threaded(const orc_case& c, const gsc::CaseConfig& cfg, unsigned threads,
                                                  double* abstraction_ms) {
    gsc::PreparedCase<std::uint32_t> p;
    p.state_grid = gsc::build_state_grid<std::uint32_t>(cfg.state_lb, cfg.state_ub, cfg.state_eta, cfg.wrap_dim);
    p.input_grid = gsc::build_input_grid(cfg.input_lb, cfg.input_ub, cfg.input_eta);
    p.model.sample_time = cfg.sample_time;
    p.model.integration_substeps = cfg.integration_substeps;
    for (int d = 0; d < 4; ++d) p.model.disturbance_half_width[d] = cfg.disturbance_half_width[d];
    p.valid_mask = gsc::build_valid_mask(p.state_grid, cfg);
    p.candidate_mask = gsc::build_candidate_mask(p.state_grid, cfg.candidate);
    overwrite_candidate(c, p);
    const std::uint64_t S = p.state_grid.total_size;
    const std::uint64_t M = p.input_grid.total_size;
    auto& a = p.abstraction;
    a.pair_count = S * M;
    a.min_flat.assign(a.pair_count, 0);
    a.max_flat.assign(a.pair_count, 0);
    a.valid.assign(a.pair_count, 0);
    const auto t0 = Clock::now();
    auto worker = [&](unsigned t) {
        for (std::uint64_t state = S * t / threads; state < S * (t + 1) / threads; ++state) {
            double x[4];
            p.state_grid.center(static_cast<std::uint32_t>(state), x);
            if (cfg.constraint_type != gsc::ConstraintType::kNone && !gsc::satisfies_state_constraint(cfg, x)) continue;
            for (std::uint64_t input = 0; input < M; ++input) {
                double u[2], mn[4], mx[4];
                p.input_grid.center(static_cast<gsc::InputIndex>(input), u);
                p.model.successor_box(x, u, p.state_grid.eta, mn, mx);
                gsc::IndexBox4D box{};
                if (!gsc::continuous_box_to_index_box(p.state_grid, mn, mx, &box)) continue;
                if (!gsc::box_satisfies_constraint(p.state_grid, box, cfg)) continue;
                const std::uint64_t pair = state * M + input;
                a.min_flat[pair] = p.state_grid.flatten(box.min);
                a.max_flat[pair] = p.state_grid.flatten(box.max);
                a.valid[pair] = 1;
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t) pool.emplace_back(worker, t);
    for (auto& th : pool) th.join();
    *abstraction_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    p.budget = gsc::estimate_memory_budget(p.state_grid, p.input_grid);
    return p;
}

// Full-grid fixpoint iterations of the reference's CPU method, timed one by
// one.  Every step starts from the solve's initial state (reachable =
// candidates, no controller: reachability.hpp:36-51), so every step does the
// same work: the reachable prefix build and every state's body
// (reachability.hpp:53-109), with the states split over threads in contiguous
// ranges.  prefix_valid is built once before the steps, as the reference
// builds it once before its loop (reachability.hpp:49).
int run_bench(const orc_case& c, unsigned threads, unsigned warmup, unsigned steps, bool single) {
    const auto cfg = to_config(c);
    double abs_ms = 0.0;
    const auto p = prepare_threaded(c, cfg, threads, &abs_ms);
    const auto& grid = p.state_grid;
    const std::uint64_t S = grid.total_size;
    const std::uint64_t M = p.input_grid.total_size;
    std::uint64_t valid_pairs = 0;
    for (auto v : p.abstraction.valid) valid_pairs += v;
    std::printf("SETUP states=%llu inputs=%llu threads=%u abstraction_ms=%.3f valid_pairs=%llu\n",
                static_cast<unsigned long long>(S), static_cast<unsigned long long>(M), threads, abs_ms,
                static_cast<unsigned long long>(valid_pairs));
    std::fflush(stdout);
    const auto prefix_valid = gsc::build_prefix_sum_cpu(grid, p.valid_mask);
    std::vector<std::uint32_t> controller(S);
    std::vector<std::uint32_t> reach_step(S);
    for (unsigned k = 0; k < warmup + steps; ++k) {
        std::fill(controller.begin(), controller.end(), gsc::kInvalidInput);
        std::fill(reach_step.begin(), reach_step.end(), gsc::kUnreachableStep);
        const std::vector<std::uint8_t>& reach = p.candidate_mask;
        std::atomic<std::uint64_t> new_reachable{0}, new_certified{0};
        const auto t0 = Clock::now();
        const auto prefix_reachable = gsc::build_prefix_sum_cpu(grid, reach);
        auto reach_next = reach;
        const auto t1 = Clock::now();
        auto worker = [&](unsigned t) {
            std::uint64_t nr = 0, nc = 0;
            for (std::uint64_t state = S * t / threads; state < S * (t + 1) / threads; ++state) {
                if (!p.valid_mask[state]) continue;
                const bool is_candidate = p.candidate_mask[state] != 0;
                const bool already_reached = reach[state] != 0;
                const bool already_certified = controller[state] != gsc::kInvalidInput;
                if ((!is_candidate && already_reached) || (is_candidate && already_certified)) continue;
                const std::uint64_t base = state * M;
                for (std::uint64_t input = 0; input < M; ++input) {
                    const std::uint64_t pair = base + input;
                    if (!p.abstraction.valid[pair]) continue;
                    const auto vc = gsc::query_box_count(grid, prefix_valid, p.abstraction.min_flat[pair],
                                                         p.abstraction.max_flat[pair]);
                    if (vc == 0) continue;
                    const auto rc = gsc::query_box_count(grid, prefix_reachable, p.abstraction.min_flat[pair],
                                                         p.abstraction.max_flat[pair]);
                    if (rc == vc) {
                        if (!already_reached) {
                            reach_next[state] = 1;
                            ++nr;
                        }
                        if (!already_certified) {
                            controller[state] = static_cast<gsc::InputIndex>(input);
                            if (is_candidate)
                                ++nc;
                            else
                                reach_step[state] = 1;
                        }
                        break;
                    }
                }
            }
            new_reachable += nr;
            new_certified += nc;
        };
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < threads; ++t) pool.emplace_back(worker, t);
        for (auto& th : pool) th.join();
        const auto t2 = Clock::now();
        std::printf("STEP k=%u warm=%d prefix_ms=%.3f states_ms=%.3f step_ms=%.3f new_reachable=%llu "
                    "new_certified=%llu\n",
                    k, k < warmup ? 1 : 0, std::chrono::duration<double, std::milli>(t1 - t0).count(),
                    std::chrono::duration<double, std::milli>(t2 - t1).count(),
                    std::chrono::duration<double, std::milli>(t2 - t0).count(),
                    static_cast<unsigned long long>(new_reachable.load()),
                    static_cast<unsigned long long>(new_certified.load()));
        std::fflush(stdout);
    }
    if (single) {
        // One iteration of the reference's own solver, single-threaded as shipped.
        const auto r = gsc::solve_backward_cpu(p, 1, false);
        std::printf("SINGLE solve_ms=%.3f iterations=%u reachable=%llu certified=%llu\n", r.solve_ms, r.iterations,
                    static_cast<unsigned long long>(r.reachable_states),
                    static_cast<unsigned long long>(r.certified_candidate_states));
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc >= 4 && std::strcmp(argv[1], "full") == 0) return run_full(read_case(argv[2]), argv[3]);
        if (argc >= 6 && std::strcmp(argv[1], "sample") == 0)
            return run_sample(read_case(argv[2]), std::stoull(argv[3]), std::stoull(argv[4]),
                              static_cast<unsigned>(std::stoul(argv[5])));
        if (argc >= 7 && std::strcmp(argv[1], "bench") == 0)
            return run_bench(read_case(argv[2]), static_cast<unsigned>(std::stoul(argv[3])),
                             static_cast<unsigned>(std::stoul(argv[4])), static_cast<unsigned>(std::stoul(argv[5])),
                             std::stoul(argv[6]) != 0);
        std::fprintf(stderr,
                     "usage: gsc_ref full <case.bin> <outdir> | sample <case.bin> <n> <seed> <threads> | "
                     "bench <case.bin> <threads> <warmup> <steps> <single>\n");
        return 1;
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "error: %s\n", ex.what());
        return 1;
    }
}
