"""Closed-loop simulation of the solved controller on the device
(gsc_problem_simulate) against the reference's own step functions
(tests/golden/sim_*.npz, made by tests/golden/make_sim_golden.py) and the
CPU restatement (oracle/sim_oracle.py).  Controller lookups and stop steps
must agree exactly; states within 1e-9 (CUDA's cos, sin and atan2 against
the C library's)."""
import json
import os

import numpy as np
import pytest

import gsc_b200 as G
import gsc_cases as C
import sim_oracle as S
from helpers import golden_index

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-9


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def solved(ctx, case):
    a = G.Abstraction(ctx, case)
    p = G.Problem(ctx, a, case, G.METHOD_FUSED)
    p.solve(graph=True)
    return a, p


def test_simulation_matches_reference_fixtures(ctx):
    with open(os.path.join(HERE, "sim_index.json")) as f:
        sims = json.load(f)
    index = golden_index()
    for name in sims:
        z = np.load(os.path.join(HERE, f"sim_{name}.npz"))
        a, p = solved(ctx, index[name]["case"])
        got = p.simulate(z["x0"], int(z["steps"]), int(z["seed"]))
        assert np.array_equal(got["steps_done"], z["steps_done"]), name
        assert np.abs(got["trajectories"] - z["trajectories"]).max() <= TOL, name
        last = z["trajectories"][np.arange(len(z["x0"])), z["steps_done"]]
        assert np.abs(got["final_states"] - last).max() <= TOL, name
        p.close()
        a.close()


def test_simulation_of_published_demo_against_oracle(ctx):
    """The script's own start point and horizon (x0 = (-0.8, -0.8, -2, 0.5),
    40 steps) on the published demo's controller, plus seeded start points."""
    case = C.hyperbolic_demo_case()
    a, p = solved(ctx, case)
    ctl = p.read()["controller"]
    shape, ishape = C.grid_shape(case)
    rng = np.random.default_rng(5)
    x0 = np.vstack([[-0.8, -0.8, -2.0, 0.5], rng.uniform([-1.8, -1.8, -3.1, 0.1], [1.8, 1.8, 3.1, 1.9], (31, 4))])
    got = p.simulate(x0, 40, 42)
    traj, done = S.simulate(ctl, S.grid_of(case, shape, ishape), x0, 40, 42)
    assert np.array_equal(got["steps_done"], done)
    assert done[0] > 0 and done.max() == 40
    assert np.abs(got["trajectories"] - traj).max() <= TOL
    p.close()
    a.close()


def test_simulation_chunks_reproducible_and_summaries_only(ctx):
    """More trajectories than one device chunk: the second chunk's
    disturbances follow the global trajectory index; a run without
    trajectories gives the same final states and stop steps."""
    case = golden_index()["hyperbolic_mid_b"]["case"]
    a, p = solved(ctx, case)
    ctl = p.read()["controller"]
    shape, ishape = C.grid_shape(case)
    n, steps = 200_000, 40                     # 1,380 B per trajectory: two chunks of device buffers
    rng = np.random.default_rng(9)
    x0 = rng.uniform(case["state_lb"], case["state_ub"], (n, 4))
    full = p.simulate(x0, steps, 7)
    summ = p.simulate(x0, steps, 7, trajectories=False)
    assert np.array_equal(full["steps_done"], summ["steps_done"])
    assert np.array_equal(full["final_states"], summ["final_states"])
    pick = np.concatenate([np.arange(0, 16), np.arange(n - 16, n)])
    traj, done = S.simulate(ctl, S.grid_of(case, shape, ishape), x0[pick], steps, 7, ids=pick)
    assert np.array_equal(full["steps_done"][pick], done)
    assert np.abs(full["trajectories"][pick] - traj).max() <= TOL
    p.close()
    a.close()
