"""Regenerates the closed-loop simulation fixtures (tests/golden/sim_*.npz)
from the REFERENCE's own post-processing code, plots/postprocess_controller.py
(ControllerSimulator.get_control_input and update_state, :103-176), run where
the reference is mounted:

    python tests/golden/make_sim_golden.py [reference root]

The simulator object is filled with a golden case's controller (from the
reference's own CPU run, tests/golden/<case>.npz) and its grid instead of an
HDF5 file (h5py and scipy are stubbed when absent: only the two methods run).
The reference draws disturbances from numpy's global generator; the fixtures
use the seeded Philox stream of oracle/sim_oracle.py instead, so the device
can reproduce them.  The loop is simulate_trajectory's (:178-224).
"""
import importlib.util
import json
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gpu-inner-outer_b200"))
import gsc_cases as C  # noqa: E402
import sim_oracle as S  # noqa: E402

CASES = {"hyperbolic_mid_b": 40, "hyperbolic_mid_a": 24}
SEED = 20261203
N_RANDOM = 14
SCRIPT_X0 = [-0.8, -0.8, -2.0, 0.5]   # postprocess_controller.py main()


def load_reference(root):
    for name in ("h5py", "scipy", "scipy.io"):
        if name not in sys.modules:
            try:
                __import__(name)
            except ImportError:
                mod = types.ModuleType(name)
                if name == "scipy.io":
                    mod.savemat = lambda *a, **k: None
                sys.modules[name] = mod
    if not hasattr(sys.modules["scipy"], "io"):
        sys.modules["scipy"].io = sys.modules["scipy.io"]
    spec = importlib.util.spec_from_file_location("postprocess_controller",
                                                  os.path.join(root, "plots", "postprocess_controller.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def grid_of(case):
    shape, ishape = C.grid_shape(case)
    return {
        "state_lb": case["state_lb"], "state_ub": case["state_ub"], "state_eta": case["state_eta"],
        "shape": list(shape), "input_lb": case["input_lb"], "input_eta": case["input_eta"],
        "input_shape": list(ishape), "sample_time": case["sample_time"],
        "integration_substeps": case["integration_substeps"],
        "disturbance_half_width": case["disturbance_half_width"],
    }


def reference_simulator(pp, case, controller):
    g = grid_of(case)
    sim = object.__new__(pp.ControllerSimulator)
    sim.controller = controller
    sim.state_lb = np.array(case["state_lb"], np.float64)
    sim.state_ub = np.array(case["state_ub"], np.float64)
    sim.state_eta = np.array(case["state_eta"], np.float64)
    sim.state_shape = np.array(g["shape"], np.uint32)
    n = g["shape"]
    sim.state_strides = np.array([1, n[0], n[0] * n[1], n[0] * n[1] * n[2]], np.uint64)
    sim.state_wrap_dim = 2
    ilb, ieta = np.array(case["input_lb"]), np.array(case["input_eta"])
    ma, mw = g["input_shape"]
    sim.input_lb, sim.input_eta = ilb, ieta
    sim.input_ub = np.array(case["input_ub"])
    sim.input_shape = np.array(g["input_shape"], np.uint32)
    centers = np.zeros((ma * mw, 2))
    for j in range(ma * mw):   # InputGrid2D::center (grid.hpp:68-78), as result_io writes it
        centers[j] = [ilb[0] + (j % ma + 0.5) * ieta[0], ilb[1] + (j // ma + 0.5) * ieta[1]]
    sim.input_centers = centers
    sim.sample_time = float(case["sample_time"])
    sim.integration_substeps = int(case["integration_substeps"])
    sim.disturbance_half_width = np.array(case["disturbance_half_width"], np.float64)
    sim.invalid_input = 0xFFFFFFFF
    return sim


def run(sim, x0s, steps, seed, K, dhw):
    n = len(x0s)
    traj = np.zeros((n, steps + 1, 4))
    done = np.zeros(n, np.uint32)
    dt = sim.sample_time / sim.integration_substeps
    for t, x0 in enumerate(x0s):
        traj[t, 0] = x0
        x = np.array(x0, np.float64)
        for step in range(steps):
            u = sim.get_control_input(x)
            if u is None:
                break
            for sub in range(K):
                d = S.disturbances(seed, [t], step, sub, K, dhw)[0]
                x = sim.update_state(x, u, d, dt)
            traj[t, step + 1] = x
            done[t] += 1
    return traj, done


def main():
    # default: the reference checkout beside this repository
    here = os.path.dirname(os.path.abspath(__file__))
    root = sys.argv[1] if len(sys.argv) > 1 else os.path.normpath(os.path.join(here, "..", "..", "..", "reference"))
    pp = load_reference(root)
    with open(os.path.join(HERE, "index.json")) as f:
        index = json.load(f)
    summary = {}
    for name, steps in CASES.items():
        case = index[name]["case"]
        with np.load(os.path.join(HERE, f"{name}.npz")) as z:
            controller = z["controller"]
        sim = reference_simulator(pp, case, controller)
        rng = np.random.default_rng(SEED)
        lo = np.array(case["state_lb"]) + 0.05 * (np.array(case["state_ub"]) - np.array(case["state_lb"]))
        hi = np.array(case["state_ub"]) - 0.05 * (np.array(case["state_ub"]) - np.array(case["state_lb"]))
        # start points with a controller, so the trajectories are not empty
        x0s = [SCRIPT_X0]
        while len(x0s) < N_RANDOM + 1:
            x = rng.uniform(lo, hi)
            if sim.get_control_input(x) is not None:
                x0s.append(list(x))
        x0s = np.array(x0s)
        traj, done = run(sim, x0s, steps, SEED, int(case["integration_substeps"]), case["disturbance_half_width"])
        np.savez_compressed(os.path.join(HERE, f"sim_{name}.npz"), x0=x0s, trajectories=traj, steps_done=done,
                            seed=np.uint64(SEED), steps=np.uint32(steps))
        summary[name] = {"steps": steps, "trajectories": len(x0s), "steps_done": done.tolist()}
        print(name, done.tolist())
    with open(os.path.join(HERE, "sim_index.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
