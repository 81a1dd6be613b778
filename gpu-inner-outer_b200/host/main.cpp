// main.cpp -- gsc_b200_cli: the reference CLI (src/main.cpp:125-218) over
// libgsc_b200.
//
//   gsc_b200_cli <config.cfg> [--gpu|--compare] [--method auto|stored|fused]
//                [--no-graph] [--output DIR] [--print-config]
//
// The summary lines keep the reference's labels (main.cpp:12-38).  --output
// writes the result arrays as raw little-endian files plus summary.json (the
// HDF5 layout of result_io.cpp needs libhdf5, which this build does not link).
// There is no CPU method in the product, so --cpu is refused; --compare keeps
// the reference's exit codes (0 = every output array equal, 3 = a difference,
// 2 = no GPU run, main.cpp:189-211) but compares the two device methods: the
// reference's own 16-corner count (stored) against the fused method.
#include <sys/stat.h>

#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>

#include "gsc/config.hpp"
#include "gsc/cuda_api.hpp"
#include "gsc_b200.h"

namespace {

std::string json_array(const double* v, int n) {
    std::ostringstream o;
    o.precision(17);
    o << "[";
    for (int i = 0; i < n; ++i) o << (i ? ", " : "") << v[i];
    o << "]";
    return o.str();
}

void print_config(const gsc::CaseConfig& c) {
    std::ostringstream o;
    o.precision(17);
    o << "{\"name\": \"" << c.name << "\", \"state_lb\": " << json_array(c.state_lb, 4)
      << ", \"state_ub\": " << json_array(c.state_ub, 4) << ", \"state_eta\": " << json_array(c.state_eta, 4)
      << ", \"wrap_dim\": " << c.wrap_dim << ", \"input_lb\": " << json_array(c.input_lb, 2)
      << ", \"input_ub\": " << json_array(c.input_ub, 2) << ", \"input_eta\": " << json_array(c.input_eta, 2)
      << ", \"candidate_lb\": " << json_array(c.candidate.lb, 4)
      << ", \"candidate_ub\": " << json_array(c.candidate.ub, 4) << ", \"map_lb\": " << json_array(c.map.lb, 4)
      << ", \"map_ub\": " << json_array(c.map.ub, 4) << ", \"obstacles\": [";
    for (size_t i = 0; i < c.obstacles.size(); ++i) {
        double v[8];
        for (int d = 0; d < 4; ++d) {
            v[d] = c.obstacles[i].lb[d];
            v[4 + d] = c.obstacles[i].ub[d];
        }
        o << (i ? ", " : "") << json_array(v, 8);
    }
    const double hyp[3] = {c.hyperbolic_params.a, c.hyperbolic_params.b, c.hyperbolic_params.c};
    const double ell[2] = {c.elliptic_params.a, c.elliptic_params.b};
    const double quad[4] = {c.quadric_params.qa, c.quadric_params.qb, c.quadric_params.c, c.quadric_params.ymax};
    const double cel[5] = {c.candidate_ellipse.cx, c.candidate_ellipse.cy, c.candidate_ellipse.wx,
                           c.candidate_ellipse.wy, c.candidate_ellipse.r2};
    o << "], \"constraint_type\": " << static_cast<int>(c.constraint_type) << ", \"hyperbolic\": " << json_array(hyp, 3)
      << ", \"elliptic\": " << json_array(ell, 2) << ", \"quadric\": " << json_array(quad, 4)
      << ", \"candidate_shape\": " << static_cast<int>(c.candidate_shape)
      << ", \"candidate_ellipse\": " << json_array(cel, 5)
      << ", \"disturbance_half_width\": " << json_array(c.disturbance_half_width, 4)
      << ", \"sample_time\": " << c.sample_time << ", \"integration_substeps\": " << c.integration_substeps
      << ", \"max_iterations\": " << c.max_iterations << ", \"verbose\": " << (c.verbose ? "true" : "false") << "}";
    std::cout << o.str() << "\n";
}

template <typename T>
void dump(const std::string& path, const std::vector<T>& v) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw std::runtime_error("cannot write " + path);
    out.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

void write_results(const std::string& dir, const gsc::CaseConfig& cfg, const gsc::GpuRunReport& g) {
    ::mkdir(dir.c_str(), 0755);
    const auto& r = g.result;
    dump(dir + "/valid_mask.u8", r.valid_mask);
    dump(dir + "/candidate_mask.u8", r.candidate_mask);
    dump(dir + "/reachable_mask.u8", r.reachable_mask);
    dump(dir + "/controller.u32", r.controller);
    dump(dir + "/reach_step.u32", r.reach_step);
    std::ofstream js(dir + "/summary.json");
    js << "{\"name\": \"" << cfg.name << "\", \"shape\": [" << g.state_grid.shape[0] << ", " << g.state_grid.shape[1]
       << ", " << g.state_grid.shape[2] << ", " << g.state_grid.shape[3] << "], \"inputs\": " << g.input_grid.total_size
       << ", \"pairs\": " << g.pair_count << ", \"iterations\": " << r.iterations
       << ", \"converged\": " << (r.converged ? "true" : "false") << ", \"message\": \"" << r.message
       << "\", \"reachable_states\": " << r.reachable_states
       << ", \"certified_candidate_states\": " << r.certified_candidate_states << ", \"abstraction_ms\": "
       << g.abstraction_ms << ", \"solve_ms\": " << g.solve_ms << ", \"iterations_stats\": [";
    for (size_t i = 0; i < g.iteration_stats.size(); ++i) {
        const auto& s = g.iteration_stats[i];
        js << (i ? ", " : "") << "[" << s.iteration << ", " << s.newly_reachable << ", " << s.newly_certified << "]";
    }
    js << "]}\n";
}

void print_summary(const gsc::GpuRunReport& g, const char* label = "gpu") {
    std::uint64_t candidates = 0;
    for (auto v : g.result.candidate_mask) candidates += (v != 0);
    const auto& r = g.result;
    std::cout << "\n[" << label << "]\n";
    std::cout << "states        : " << g.state_grid.total_size << '\n';
    std::cout << "inputs        : " << g.input_grid.total_size << '\n';
    std::cout << "pairs         : " << g.pair_count << '\n';
    std::cout << "reachable     : " << r.reachable_states << '\n';
    std::cout << "candidate     : " << candidates << '\n';
    std::cout << "candidate ctl : " << r.certified_candidate_states << '\n';
    std::cout << "iterations    : " << r.iterations << '\n';
    std::cout << "converged     : " << (r.converged ? "true" : "false") << '\n';
    std::cout << "message       : " << r.message << '\n';
    std::cout << "abstraction   : " << g.abstraction_ms << " ms\n";
    std::cout << "solve         : " << g.solve_ms << " ms\n";
    std::cout << "device memory : " << g.memory_stats.total_allocated_bytes << " bytes\n";
    for (const auto& s : g.iteration_stats)
        std::cout << "  Iter " << s.iteration << ": " << s.newly_reachable << " new reachable, " << s.newly_certified
                  << " new certified\n";
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: gsc_b200_cli <config.cfg> [--gpu|--compare] [--method auto|stored|fused] "
                     "[--no-graph] [--output DIR] [--print-config]\n";
        return 1;
    }
    try {
        const std::string path = argv[1];
        gsc::RunOptions opt;
        std::string output;
        bool print_only = false;
        bool compare = false;
        for (int i = 2; i < argc; ++i) {
            const std::string a = argv[i];
            if (a == "--gpu") continue;
            if (a == "--compare") {
                compare = true;
                continue;
            }
            if (a == "--cpu") {
                std::cerr << "error: --cpu needs the CPU method, which this library does not ship\n";
                return 2;
            }
            if (a == "--no-graph") {
                opt.graph = false;
            } else if (a == "--print-config") {
                print_only = true;
            } else if (a == "--method" && i + 1 < argc) {
                const std::string m = argv[++i];
                opt.method = m == "stored" ? GSC_METHOD_STORED : m == "fused" ? GSC_METHOD_FUSED : GSC_METHOD_AUTO;
            } else if (a == "--output" && i + 1 < argc) {
                output = argv[++i];
            } else {
                throw std::runtime_error("unknown argument: " + a);
            }
        }
        const gsc::CaseConfig cfg = gsc::load_case_config(path);
        if (print_only) {
            print_config(cfg);
            return 0;
        }
        if (compare) {   // main.cpp:189-211, the two device methods
            gsc::RunOptions so = opt, fo = opt;
            so.method = GSC_METHOD_STORED;
            fo.method = GSC_METHOD_FUSED;
            const gsc::GpuRunReport s = gsc::run_case_cuda_u32(cfg, so);
            const gsc::GpuRunReport f = s.executed ? gsc::run_case_cuda_u32(cfg, fo) : s;
            if (!s.executed || !f.executed) {
                std::cerr << "gpu compare unavailable: " << (s.executed ? f.message : s.message) << '\n';
                return 2;
            }
            print_summary(s, "stored");
            print_summary(f, "fused");
            const auto& a = s.result;
            const auto& b = f.result;
            const bool same = a.valid_mask == b.valid_mask && a.candidate_mask == b.candidate_mask &&
                              a.reachable_mask == b.reachable_mask && a.controller == b.controller &&
                              a.reach_step == b.reach_step && a.iterations == b.iterations &&
                              a.message == b.message;
            if (!output.empty()) write_results(output, cfg, f);
            std::cout << "exact_match   : " << (same ? "true" : "false") << '\n';
            return same ? 0 : 3;
        }
        const gsc::GpuRunReport g = gsc::run_case_cuda_u32(cfg, opt);
        if (!g.executed) {   // main.cpp:168-171
            std::cerr << "gpu run unavailable: " << g.message << '\n';
            return 2;
        }
        print_summary(g);
        if (!output.empty()) {
            write_results(output, cfg, g);
            std::cout << "result dir    : " << output << '\n';
        }
        return 0;
    } catch (const std::exception& ex) {
        std::cerr << "error: " << ex.what() << '\n';
        return 1;
    }
}
