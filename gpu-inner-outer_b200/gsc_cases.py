"""Case descriptions for the grid symbolic-control path.

A case is a plain dict with the fields of the reference's ``CaseConfig``
(include/gsc/config.hpp:41-67) plus two extensions that the benchmark
workloads need:

* ``constraint = "quadric"`` with ``constraint_params = (qa, qb, c, ymax)``:
  the safe set ``(x*x)*qa - (y*y)*qb <= c and fabs(y) <= ymax``.  The
  reference can state it only as ``ConstraintType::kCustom`` with a predicate
  of exactly that expression (config.cpp:119-123).
* ``candidate = "ellipse"`` with ``candidate_ellipse = (cx, cy, wx, wy, r2)``:
  the candidate set ``valid and (dx*dx)*wx + (dy*dy)*wy <= r2`` with
  ``dx = x - cx, dy = y - cy``.

The reference's own built-in cases are restated from config.cpp:129-241 and
examples/hyperbolic_case.cfg.  The benchmark grids cover x, y in [-2, 2],
theta in [-pi, pi) (wrapped, dimension 2) and v in [0, 1] with
``eta = width / n``.
"""
from __future__ import annotations

import copy
import math

PI = 3.141592653589793


def default_case() -> dict:
    """make_default_case (config.cpp:129-139)."""
    return {
        "name": "unicycle_default",
        "state_lb": [-2.0, -2.0, -PI, 0.0],
        "state_ub": [2.0, 2.0, PI, 2.0],
        "state_eta": [0.5, 0.5, 0.7853981633974483, 0.5],
        "wrap_dim": 2,
        "input_lb": [-0.5, -1.0],
        "input_ub": [0.5, 1.0],
        "input_eta": [0.5, 1.0],
        "candidate": "rect",
        "candidate_lb": [-0.5, -0.5, -PI, 0.0],
        "candidate_ub": [0.5, 0.5, PI, 1.5],
        "map_lb": [-2.0, -2.0, -PI, 0.0],
        "map_ub": [2.0, 2.0, PI, 2.0],
        "obstacles": [[0.5, -0.5, -PI, 0.0, 1.0, 0.5, PI, 2.0]],
        "constraint": "none",
        "constraint_params": [0.0, 0.0, 0.0, 0.0],
        "disturbance_half_width": [0.05, 0.05, 0.02, 0.02],
        "sample_time": 0.2,
        "integration_substeps": 32,
        "max_iterations": 32,
    }


def wraparound_case() -> dict:
    """make_wraparound_case (config.cpp:141-154)."""
    c = default_case()
    c["name"] = "wraparound_case"
    c["state_eta"][2] = 0.5235987755982988
    c["disturbance_half_width"][2] = 0.35
    c["candidate_lb"] = [-0.5, -0.5, 2.6, 0.0]
    c["candidate_ub"] = [0.5, 0.5, PI, 1.5]
    c["obstacles"] = []
    return c


def smoke_case() -> dict:
    """make_smoke_case (config.cpp:156-185)."""
    c = default_case()
    c.update({
        "name": "smoke_case",
        "state_lb": [-6.0, -6.0, -PI, 0.0],
        "state_ub": [6.0, 6.0, PI, 4.0],
        "state_eta": [0.3, 0.3, 0.39269908169872414, 0.5],
        "input_lb": [-1.0, -1.5],
        "input_ub": [1.0, 1.5],
        "input_eta": [0.25, 0.3],
        "candidate_lb": [-1.0, -1.0, -PI, 0.0],
        "candidate_ub": [1.0, 1.0, PI, 2.0],
        "obstacles": [],
        "max_iterations": 4,
    })
    c["map_lb"] = list(c["state_lb"])
    c["map_ub"] = list(c["state_ub"])
    return c


def hyperbolic_demo_case() -> dict:
    """examples/hyperbolic_case.cfg as read by load_case_config (config.cpp:243-347):
    the published demo run, 70x70x63x13 states x 100 inputs."""
    return {
        "name": "hyperbolic_demo",
        "state_lb": [-3.5, -3.5, -PI, -0.1],
        "state_ub": [3.5, 3.5, PI, 1.1],
        "state_eta": [0.1, 0.1, 0.1, 0.1],
        "wrap_dim": 2,
        "input_lb": [-1.0, -1.0],
        "input_ub": [1.0, 1.0],
        "input_eta": [0.2, 0.2],
        "candidate": "rect",
        "candidate_lb": [-0.8, -0.8, -PI, 0.0],
        "candidate_ub": [0.8, 0.8, PI, 1.0],
        "map_lb": [-3.5, -3.5, -PI, -0.1],
        "map_ub": [3.5, 3.5, PI, 1.1],
        "obstacles": [],
        "constraint": "hyperbolic",
        "constraint_params": [4.0, 4.0, 16.0, 0.0],
        "disturbance_half_width": [0.05, 0.05, 0.05, 0.05],
        "sample_time": 0.5,
        "integration_substeps": 32,
        "max_iterations": 100,
    }


def unicycle_grid_case(n, m, name=None, max_iterations=256) -> dict:
    """The benchmark family: grid n = (nx, ny, ntheta, nv) over x, y in [-2, 2],
    theta in [-pi, pi), v in [0, 1]; inputs m = (m_a, m_omega) over
    a in [-0.5, 0.5] (input dim 0) and omega in [-1, 1] (input dim 1);
    tau = 0.1 s, one Euler step, disturbance 0.01 per dimension; safe set
    x^2 - y^2 <= 1 and |y| <= 1.8; candidate x^2 + y^2 <= 0.5 within the
    valid set."""
    lb = [-2.0, -2.0, -PI, 0.0]
    ub = [2.0, 2.0, PI, 1.0]
    ilb = [-0.5, -1.0]
    iub = [0.5, 1.0]
    c = {
        "name": name or f"unicycle_{n[0]}x{n[1]}x{n[2]}x{n[3]}_{m[0]}x{m[1]}",
        "state_lb": lb,
        "state_ub": ub,
        "state_eta": [(ub[d] - lb[d]) / n[d] for d in range(4)],
        "wrap_dim": 2,
        "input_lb": ilb,
        "input_ub": iub,
        "input_eta": [(iub[d] - ilb[d]) / m[d] for d in range(2)],
        "candidate": "ellipse",
        "candidate_ellipse": [0.0, 0.0, 1.0, 1.0, 0.5],
        "map_lb": list(lb),
        "map_ub": list(ub),
        "obstacles": [],
        "constraint": "quadric",
        "constraint_params": [1.0, 1.0, 1.0, 1.8],
        "disturbance_half_width": [0.01, 0.01, 0.01, 0.01],
        "sample_time": 0.1,
        "integration_substeps": 1,
        "max_iterations": max_iterations,
        "expect_shape": list(n),
        "expect_input_shape": list(m),
    }
    return c


def small_case() -> dict:
    """20x20x16x10 states x 5x5 inputs (64,000 cells, 1.6 M pairs)."""
    return unicycle_grid_case((20, 20, 16, 10), (5, 5), "unicycle_small_20x20x16x10_5x5")


def demo_scale_case() -> dict:
    """65x65x38x25 states x 10x10 inputs (4,013,750 cells, 401,375,000 pairs)."""
    return unicycle_grid_case((65, 65, 38, 25), (10, 10), "unicycle_demo_scale_65x65x38x25_10x10")


def large_case() -> dict:
    """128x128x72x48 states x 12x12 inputs (56,623,104 cells, 8.15 G pairs)."""
    return unicycle_grid_case((128, 128, 72, 48), (12, 12), "unicycle_large_128x128x72x48_12x12")


def serve_mid_case() -> dict:
    """32x32x24x16 states x 8x8 inputs (the third resident serving grid)."""
    return unicycle_grid_case((32, 32, 24, 16), (8, 8), "unicycle_serve_32x32x24x16_8x8")


def grid_shape(case):
    """build_state_grid / build_input_grid shapes (grid.hpp:103-168)."""
    s = tuple(int(math.ceil((case["state_ub"][d] - case["state_lb"][d]) / case["state_eta"][d]))
              for d in range(4))
    u = tuple(int(math.ceil((case["input_ub"][d] - case["input_lb"][d]) / case["input_eta"][d]))
              for d in range(2))
    return s, u


def checked(case: dict) -> dict:
    """Return the case after asserting that eta = width / n gave the intended shape."""
    s, u = grid_shape(case)
    if "expect_shape" in case and list(s) != list(case["expect_shape"]):
        raise ValueError(f"grid shape {s} != intended {case['expect_shape']}")
    if "expect_input_shape" in case and list(u) != list(case["expect_input_shape"]):
        raise ValueError(f"input shape {u} != intended {case['expect_input_shape']}")
    return case


def clone(case: dict, **over) -> dict:
    c = copy.deepcopy(case)
    c.update(over)
    return c


PRESETS = {
    "default": default_case,
    "wraparound": wraparound_case,
    "smoke": smoke_case,
    "hyperbolic_demo": hyperbolic_demo_case,
    "small": small_case,
    "demo_scale": demo_scale_case,
    "large": large_case,
    "serve_mid": serve_mid_case,
}


def random_instance(seed: int, index: int, n_lo=(16, 16, 16, 16), n_hi=(48, 48, 32, 24), m_lo=(5, 5),
                    m_hi=(10, 10), max_iterations=256) -> dict:
    """One seeded instance of the batched workload: grid n_d in [n_lo_d, n_hi_d],
    inputs m_a x m_omega in [25, 100], tau in U[0.05, 0.2], disturbance bound in
    U[0.005, 0.02], safe set x^2/alpha - y^2/beta <= 1 and |y| <= gamma, and an
    elliptical candidate set centred inside it, intersected with the valid set."""
    import numpy as np

    rng = np.random.default_rng([int(seed), int(index)])
    lb = [-2.0, -2.0, -PI, 0.0]
    ub = [2.0, 2.0, PI, 1.0]
    n = []
    for d in range(4):
        while True:
            k = int(rng.integers(n_lo[d], n_hi[d] + 1))
            eta = (ub[d] - lb[d]) / k
            if int(math.ceil((ub[d] - lb[d]) / eta)) == k:
                n.append(k)
                break
    m = [int(rng.integers(m_lo[d], m_hi[d] + 1)) for d in range(2)]
    c = unicycle_grid_case(tuple(n), tuple(m), f"instance_{seed}_{index}", max_iterations)
    c["sample_time"] = float(rng.uniform(0.05, 0.2))
    dhw = float(rng.uniform(0.005, 0.02))
    c["disturbance_half_width"] = [dhw] * 4
    alpha = float(rng.uniform(0.5, 2.0))
    beta = float(rng.uniform(0.5, 2.0))
    gamma = float(rng.uniform(1.2, 1.9))
    c["constraint_params"] = [1.0 / alpha, 1.0 / beta, 1.0, gamma]
    cx, cy = (float(v) for v in rng.uniform(-0.5, 0.5, size=2))
    ax, ay = (float(v) for v in rng.uniform(0.3, 0.8, size=2))
    c["candidate_ellipse"] = [cx, cy, 1.0 / (ax * ax), 1.0 / (ay * ay), 1.0]
    return checked(c)


def random_query(case: dict, seed: int, index: int, iter_lo=8, iter_hi=64) -> dict:
    """One seeded K-invariance query against the model of `case` (same grid,
    inputs and dynamics): safe set x^2/alpha - y^2/beta <= 1 and |y| <= gamma,
    an elliptical candidate set centred inside it (within the valid set), a
    disturbance bound in U[0.005, 0.02] on every dimension, and an iteration
    cap in [iter_lo, iter_hi]."""
    import numpy as np

    rng = np.random.default_rng([int(seed), int(index), 7])
    q = clone(case)
    q["name"] = f"{case['name']}_q{seed}_{index}"
    q["disturbance_half_width"] = [float(rng.uniform(0.005, 0.02))] * 4
    alpha = float(rng.uniform(0.5, 2.0))
    beta = float(rng.uniform(0.5, 2.0))
    gamma = float(rng.uniform(1.2, 1.9))
    q["constraint"] = "quadric"
    q["constraint_params"] = [1.0 / alpha, 1.0 / beta, 1.0, gamma]
    cx, cy = (float(v) for v in rng.uniform(-0.5, 0.5, size=2))
    ax, ay = (float(v) for v in rng.uniform(0.3, 0.8, size=2))
    q["candidate"] = "ellipse"
    q["candidate_ellipse"] = [cx, cy, 1.0 / (ax * ax), 1.0 / (ay * ay), 1.0]
    q["max_iterations"] = int(rng.integers(iter_lo, iter_hi + 1))
    return q
