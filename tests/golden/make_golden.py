"""Regenerates the golden fixtures of tests/golden from the REFERENCE's own CPU
method (oracle/_ref/gsc_ref, compiled by oracle/Makefile from the reference's
sources).  Run from the repository root where the reference is mounted:

    make -C oracle && python tests/golden/make_golden.py

Each case is written as <name>.npz (masks, controller, reach_step and
per-iteration counts as the reference produced them) and summarised in
index.json with SHA-256 digests of every array, including the per-pair
abstraction (min_flat, max_flat, valid; abstraction.hpp:161-209), whose full
arrays are kept only for the smallest cases.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gpu-inner-outer_b200"))
import gsc_cases as C  # noqa: E402
import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
FULL_ABSTRACTION_MAX_PAIRS = 1 << 15


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden_cases():
    cases = {
        "default": C.default_case(),
        "wraparound": C.wraparound_case(),
        "small": C.small_case(),
        "smoke": C.smoke_case(),
    }
    c = C.default_case()
    c.update(name="default_elliptic", constraint="elliptic", constraint_params=[1.8, 1.6, 0.0, 0.0])
    cases["default_elliptic"] = c
    c = C.hyperbolic_demo_case()
    c.update(name="hyperbolic_coarse", state_eta=[0.35, 0.35, 0.35, 0.3], input_eta=[0.4, 0.4],
             integration_substeps=8, max_iterations=50)
    cases["hyperbolic_coarse"] = c
    c = C.small_case()
    c.update(name="small_maxiter0", max_iterations=0)
    cases["small_maxiter0"] = c
    c = C.default_case()
    c.update(name="default_empty_candidate", candidate_lb=[3.0, 3.0, 0.0, 0.0], candidate_ub=[4.0, 4.0, 0.0, 0.0])
    cases["default_empty_candidate"] = c
    c = C.wraparound_case()
    c.update(name="wraparound_full_circle")
    c["disturbance_half_width"] = [0.05, 0.05, 20.0, 0.02]
    cases["wraparound_full_circle"] = c
    c = C.small_case()
    c.update(name="small_obstacles", obstacles=[[0.8, -0.4, -C.PI, 0.0, 1.2, 0.4, C.PI, 1.0],
                                                [-1.5, 0.6, -1.0, 0.2, -0.9, 1.2, 1.0, 0.8]],
             max_iterations=6)
    cases["small_obstacles"] = c
    c = C.small_case()
    c.update(name="small_hyperbolic_rect", constraint="hyperbolic", constraint_params=[1.0, 0.5, 2.0, 0.0],
             candidate="rect", candidate_lb=[-0.6, -0.6, -C.PI, 0.0], candidate_ub=[0.6, 0.6, C.PI, 1.0])
    cases["small_hyperbolic_rect"] = c
    c = C.hyperbolic_demo_case()
    c.update(name="hyperbolic_mid_a", state_eta=[0.2, 0.2, 0.2, 0.2], input_eta=[0.4, 0.4])
    cases["hyperbolic_mid_a"] = c     # 35x35x32x7 x 25 inputs, 32 substeps: 14 iterations
    c = C.hyperbolic_demo_case()
    c.update(name="hyperbolic_mid_b", state_eta=[0.2, 0.2, 0.15, 0.15], input_eta=[0.5, 0.5],
             integration_substeps=8)
    cases["hyperbolic_mid_b"] = c     # 35x35x42x9 x 16 inputs: 34 iterations
    for i in range(4):
        c = C.random_instance(20261203, i, n_lo=(8, 8, 8, 6), n_hi=(24, 24, 16, 12))
        c["name"] = f"mini_instance_{i}"
        cases[c["name"]] = c
    return cases


def main():
    index = {}
    for name, case in golden_cases().items():
        r = O.run_reference(case)
        mn = r.pop("min_flat", None)
        mx = r.pop("max_flat", None)
        pv = r.pop("pair_valid", None)
        arrays = {k: r[k] for k in ("valid_mask", "candidate_mask", "reachable_mask", "controller", "reach_step",
                                   "iter_new_reachable", "iter_new_certified")}
        entry = {
            "case": case,
            "iterations": int(r["iterations"]),
            "converged": bool(r["converged"]),
            "message": r["message"],
            "reachable_states": int(r["reachable_states"]),
            "certified_candidates": int(r["certified_candidates"]),
            "valid_pairs": int(r["valid_pairs"]),
            "sha256": {k: sha(v) for k, v in arrays.items() if k.startswith(("valid", "cand", "reach", "contr"))},
        }
        if mn is not None:
            entry["abstraction_sha256"] = {"min_flat": sha(mn), "max_flat": sha(mx), "valid": sha(pv)}
            if mn.size <= FULL_ABSTRACTION_MAX_PAIRS:
                arrays.update(min_flat=mn, max_flat=mx, pair_valid=pv)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        index[name] = entry
        print(name, entry["iterations"], entry["reachable_states"], entry["message"], flush=True)
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
