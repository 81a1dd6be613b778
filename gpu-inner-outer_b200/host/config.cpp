// config.cpp -- case descriptions and the .cfg parser of the gsc host API.
//
// Behaviour follows the reference's src/config.cpp: the predicates of
// config.cpp:62-127, the built-in cases of :129-241 and the key = value
// format of :243-347 ('#' starts a comment, blank lines are skipped, unknown
// keys are an error, the map defaults to the state bounds).
#include "gsc/config.hpp"

#include <cctype>
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace gsc {

namespace {

constexpr double kPi = 3.141592653589793;

std::string strip(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) ++b;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) --e;
    return s.substr(b, e - b);
}

std::vector<double> numbers(const std::string& value) {
    std::vector<double> out;
    std::stringstream in(value);
    std::string item;
    while (std::getline(in, item, ',')) out.push_back(std::stod(strip(item)));
    return out;
}

void take(const std::vector<double>& v, double* dst, size_t n, const std::string& key) {
    if (v.size() != n)
        throw std::runtime_error(key + " expects " + std::to_string(n) + " comma-separated numbers");
    for (size_t i = 0; i < n; ++i) dst[i] = v[i];
}

HyperRect4D rect(const double lb[4], const double ub[4]) {
    HyperRect4D r;
    for (int d = 0; d < 4; ++d) {
        r.lb[d] = lb[d];
        r.ub[d] = ub[d];
    }
    return r;
}

}  // namespace

bool point_in_rect(const HyperRect4D& r, const double x[kStateDim]) {
    for (int d = 0; d < kStateDim; ++d)
        if (x[d] < r.lb[d] || x[d] > r.ub[d]) return false;
    return true;
}

bool satisfies_state_constraint(const CaseConfig& cfg, const double x[kStateDim]) {
    switch (cfg.constraint_type) {
        case ConstraintType::kHyperbolic: {
            const double xx = x[0] * x[0], yy = x[1] * x[1];
            return (xx - yy <= cfg.hyperbolic_params.a) && (cfg.hyperbolic_params.b * yy - xx <= cfg.hyperbolic_params.c);
        }
        case ConstraintType::kElliptic: {
            const double u = x[0] / cfg.elliptic_params.a, v = x[1] / cfg.elliptic_params.b;
            return u * u + v * v <= 1.0;
        }
        case ConstraintType::kQuadric: {
            const QuadricConstraintParams& p = cfg.quadric_params;
            return ((x[0] * x[0]) * p.qa - (x[1] * x[1]) * p.qb <= p.c) && (std::fabs(x[1]) <= p.ymax);
        }
        case ConstraintType::kCustom:
            return cfg.custom_constraint ? cfg.custom_constraint(x) : true;
        default:
            return true;
    }
}

CaseConfig make_default_case() {
    CaseConfig cfg;
    const double clb[4] = {-0.5, -0.5, -kPi, 0.0}, cub[4] = {0.5, 0.5, kPi, 1.5};
    cfg.candidate = rect(clb, cub);
    cfg.map = rect(cfg.state_lb, cfg.state_ub);
    const double olb[4] = {0.5, -0.5, -kPi, 0.0}, oub[4] = {1.0, 0.5, kPi, 2.0};
    cfg.obstacles.push_back(rect(olb, oub));
    return cfg;
}

CaseConfig make_wraparound_case() {
    CaseConfig cfg = make_default_case();
    cfg.name = "wraparound_case";
    cfg.state_eta[2] = 0.5235987755982988;
    cfg.disturbance_half_width[2] = 0.35;
    const double clb[4] = {-0.5, -0.5, 2.6, 0.0}, cub[4] = {0.5, 0.5, kPi, 1.5};
    cfg.candidate = rect(clb, cub);
    cfg.map = rect(cfg.state_lb, cfg.state_ub);
    cfg.obstacles.clear();
    return cfg;
}

CaseConfig make_smoke_case() {
    CaseConfig cfg = make_default_case();
    cfg.name = "smoke_case";
    const double lb[4] = {-6.0, -6.0, -kPi, 0.0}, ub[4] = {6.0, 6.0, kPi, 4.0};
    const double eta[4] = {0.3, 0.3, 0.39269908169872414, 0.5};
    for (int d = 0; d < 4; ++d) {
        cfg.state_lb[d] = lb[d];
        cfg.state_ub[d] = ub[d];
        cfg.state_eta[d] = eta[d];
    }
    cfg.input_lb[0] = -1.0;
    cfg.input_ub[0] = 1.0;
    cfg.input_eta[0] = 0.25;
    cfg.input_lb[1] = -1.5;
    cfg.input_ub[1] = 1.5;
    cfg.input_eta[1] = 0.3;
    const double clb[4] = {-1.0, -1.0, -kPi, 0.0}, cub[4] = {1.0, 1.0, kPi, 2.0};
    cfg.candidate = rect(clb, cub);
    cfg.map = rect(cfg.state_lb, cfg.state_ub);
    cfg.obstacles.clear();
    cfg.max_iterations = 4;
    cfg.verbose = false;
    return cfg;
}

CaseConfig make_hyperbolic_case() {
    CaseConfig cfg;
    cfg.name = "hyperbolic_case";
    const double lb[4] = {-3.5, -3.5, -kPi, 0.2}, ub[4] = {3.5, 3.5, kPi, 2.0}, eta[4] = {0.1, 0.1, 0.1, 0.2};
    for (int d = 0; d < 4; ++d) {
        cfg.state_lb[d] = lb[d];
        cfg.state_ub[d] = ub[d];
        cfg.state_eta[d] = eta[d];
    }
    cfg.wrap_dim = 2;
    cfg.input_lb[0] = 0.2;
    cfg.input_ub[0] = 2.0;
    cfg.input_lb[1] = -1.0;
    cfg.input_ub[1] = 1.0;
    cfg.input_eta[0] = 0.3;
    cfg.input_eta[1] = 0.4;
    const double clb[4] = {-1.0, -1.0, -kPi, 0.2}, cub[4] = {1.0, 1.0, kPi, 2.0};
    cfg.candidate = rect(clb, cub);
    cfg.map = rect(cfg.state_lb, cfg.state_ub);
    cfg.constraint_type = ConstraintType::kHyperbolic;
    cfg.hyperbolic_params = {4.0, 4.0, 16.0};
    const double dhw[4] = {0.12, 0.12, 0.12, 0.0};
    for (int d = 0; d < 4; ++d) cfg.disturbance_half_width[d] = dhw[d];
    cfg.sample_time = 1.0;
    cfg.integration_substeps = 32;
    cfg.max_iterations = 100;
    return cfg;
}

CaseConfig make_unicycle_grid_case(const std::uint32_t n[4], const std::uint32_t m[2]) {
    CaseConfig cfg;
    cfg.name = "unicycle_" + std::to_string(n[0]) + "x" + std::to_string(n[1]) + "x" + std::to_string(n[2]) + "x" +
               std::to_string(n[3]) + "_" + std::to_string(m[0]) + "x" + std::to_string(m[1]);
    const double lb[4] = {-2.0, -2.0, -kPi, 0.0}, ub[4] = {2.0, 2.0, kPi, 1.0};
    for (int d = 0; d < 4; ++d) {
        cfg.state_lb[d] = lb[d];
        cfg.state_ub[d] = ub[d];
        cfg.state_eta[d] = (ub[d] - lb[d]) / n[d];
        cfg.disturbance_half_width[d] = 0.01;
    }
    cfg.input_lb[0] = -0.5;
    cfg.input_ub[0] = 0.5;
    cfg.input_lb[1] = -1.0;
    cfg.input_ub[1] = 1.0;
    for (int d = 0; d < 2; ++d) cfg.input_eta[d] = (cfg.input_ub[d] - cfg.input_lb[d]) / m[d];
    cfg.map = rect(cfg.state_lb, cfg.state_ub);
    cfg.constraint_type = ConstraintType::kQuadric;
    cfg.quadric_params = {1.0, 1.0, 1.0, 1.8};
    cfg.candidate_shape = CandidateShape::kEllipse;
    cfg.candidate_ellipse = {0.0, 0.0, 1.0, 1.0, 0.5};
    cfg.sample_time = 0.1;
    cfg.integration_substeps = 1;
    cfg.max_iterations = 256;
    return cfg;
}

CaseConfig parse_case_config(const std::string& text) {
    CaseConfig cfg = make_default_case();
    cfg.obstacles.clear();
    std::stringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        line = strip(line);
        if (line.empty()) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) throw std::runtime_error("expected key=value line: " + line);
        const std::string key = strip(line.substr(0, eq));
        const std::string value = strip(line.substr(eq + 1));
        if (key == "name") cfg.name = value;
        else if (key == "state_lb") take(numbers(value), cfg.state_lb, 4, key);
        else if (key == "state_ub") take(numbers(value), cfg.state_ub, 4, key);
        else if (key == "state_eta") take(numbers(value), cfg.state_eta, 4, key);
        else if (key == "wrap_dim") cfg.wrap_dim = std::stoi(value);
        else if (key == "input_lb") take(numbers(value), cfg.input_lb, 2, key);
        else if (key == "input_ub") take(numbers(value), cfg.input_ub, 2, key);
        else if (key == "input_eta") take(numbers(value), cfg.input_eta, 2, key);
        else if (key == "candidate_lb") take(numbers(value), cfg.candidate.lb, 4, key);
        else if (key == "candidate_ub") take(numbers(value), cfg.candidate.ub, 4, key);
        else if (key == "map_lb") take(numbers(value), cfg.map.lb, 4, key);
        else if (key == "map_ub") take(numbers(value), cfg.map.ub, 4, key);
        else if (key == "disturbance_half_width") take(numbers(value), cfg.disturbance_half_width, 4, key);
        else if (key == "sample_time") cfg.sample_time = std::stod(value);
        else if (key == "integration_substeps") cfg.integration_substeps = static_cast<std::uint32_t>(std::stoul(value));
        else if (key == "max_iterations") cfg.max_iterations = static_cast<std::uint32_t>(std::stoul(value));
        else if (key == "verbose") cfg.verbose = (value == "1" || value == "true" || value == "TRUE");
        else if (key == "obstacle") {
            const auto v = numbers(value);
            if (v.size() != 8) throw std::runtime_error("obstacle expects 8 comma-separated numbers");
            HyperRect4D r;
            for (int d = 0; d < 4; ++d) {
                r.lb[d] = v[d];
                r.ub[d] = v[4 + d];
            }
            cfg.obstacles.push_back(r);
        } else if (key == "constraint_type") {
            if (value == "none") cfg.constraint_type = ConstraintType::kNone;
            else if (value == "hyperbolic") cfg.constraint_type = ConstraintType::kHyperbolic;
            else if (value == "elliptic") cfg.constraint_type = ConstraintType::kElliptic;
            else if (value == "quadric") cfg.constraint_type = ConstraintType::kQuadric;
            else throw std::runtime_error("unknown constraint_type: " + value);
        } else if (key == "hyperbolic_a") cfg.hyperbolic_params.a = std::stod(value);
        else if (key == "hyperbolic_b") cfg.hyperbolic_params.b = std::stod(value);
        else if (key == "hyperbolic_c") cfg.hyperbolic_params.c = std::stod(value);
        else if (key == "elliptic_a") cfg.elliptic_params.a = std::stod(value);
        else if (key == "elliptic_b") cfg.elliptic_params.b = std::stod(value);
        else if (key == "quadric_qa") cfg.quadric_params.qa = std::stod(value);
        else if (key == "quadric_qb") cfg.quadric_params.qb = std::stod(value);
        else if (key == "quadric_c") cfg.quadric_params.c = std::stod(value);
        else if (key == "quadric_ymax") cfg.quadric_params.ymax = std::stod(value);
        else if (key == "candidate_shape") {
            if (value == "rect") cfg.candidate_shape = CandidateShape::kRect;
            else if (value == "ellipse") cfg.candidate_shape = CandidateShape::kEllipse;
            else throw std::runtime_error("unknown candidate_shape: " + value);
        } else if (key == "candidate_ellipse") {
            double e[5];
            take(numbers(value), e, 5, key);
            cfg.candidate_ellipse = {e[0], e[1], e[2], e[3], e[4]};
        } else {
            throw std::runtime_error("unknown config key: " + key);
        }
    }
    if (cfg.map.ub[0] == 0.0 && cfg.map.lb[0] == 0.0) cfg.map = rect(cfg.state_lb, cfg.state_ub);
    return cfg;
}

CaseConfig load_case_config(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("failed to open config: " + path);
    std::stringstream buf;
    buf << in.rdbuf();
    return parse_case_config(buf.str());
}

}  // namespace gsc
