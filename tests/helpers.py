"""Shared helpers for the tests: golden fixtures and exact comparisons."""
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

ARRAYS = ("valid_mask", "candidate_mask", "reachable_mask", "controller", "reach_step")


def golden_index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def golden_arrays(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def assert_same_result(got, want, label=""):
    """Bit-exact comparison of the reference outputs (main.cpp:114-121 same_result,
    plus iteration count, stop message and per-iteration counts)."""
    for k in ARRAYS:
        g = np.asarray(got[k])
        w = np.asarray(want[k])
        assert g.dtype == w.dtype and g.shape == w.shape, f"{label} {k}: {g.dtype}{g.shape} vs {w.dtype}{w.shape}"
        if not np.array_equal(g, w):
            bad = np.flatnonzero(g != w)
            raise AssertionError(f"{label} {k}: {bad.size} mismatches, first at {bad[:5]}: "
                                 f"got {g[bad[:5]]} want {w[bad[:5]]}")
    for k in ("iter_new_reachable", "iter_new_certified"):
        if k in want and k in got:
            assert list(np.asarray(got[k], dtype=np.uint64)) == list(np.asarray(want[k], dtype=np.uint64)), \
                f"{label} {k}"
