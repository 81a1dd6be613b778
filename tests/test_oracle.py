"""The CPU oracle against the reference: golden fixtures produced by the
reference's own CPU method (tests/golden/make_golden.py) and the reference's
published demo run (README.md:44-98)."""
import hashlib

import numpy as np
import pytest

import gsc_cases as C
import oracle as O
from helpers import assert_same_result, golden_arrays, golden_index

INDEX = golden_index()


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(INDEX))
def test_oracle_matches_reference_golden(name):
    entry = INDEX[name]
    got = O.solve(entry["case"])
    want = golden_arrays(name)
    assert_same_result(got, want, name)
    assert got["iterations"] == entry["iterations"]
    assert got["converged"] == entry["converged"]
    assert got["message"] == entry["message"]
    assert got["reachable_states"] == entry["reachable_states"]
    assert got["certified_candidates"] == entry["certified_candidates"]
    assert got["valid_pairs"] == entry["valid_pairs"]


@pytest.mark.parametrize("name", sorted(INDEX))
def test_oracle_abstraction_matches_reference(name):
    entry = INDEX[name]
    if "abstraction_sha256" not in entry:
        pytest.skip("abstraction not dumped for this size")
    mn, mx, pv = O.abstraction(entry["case"])
    assert sha(mn) == entry["abstraction_sha256"]["min_flat"]
    assert sha(mx) == entry["abstraction_sha256"]["max_flat"]
    assert sha(pv) == entry["abstraction_sha256"]["valid"]


def test_oracle_reproduces_published_demo():
    """examples/hyperbolic_case.cfg: README.md:44-98 (counts) and the reference
    CPU outputs' SHA-256 prefixes."""
    o = O.solve(C.hyperbolic_demo_case())
    assert o["states"] == 4013100 and o["inputs"] == 100 and o["pairs"] == 401310000
    assert o["reachable_states"] == 1142689
    assert o["candidate_count"] == 161280 and o["certified_candidates"] == 161280
    assert o["iterations"] == 12 and o["converged"]
    assert o["message"] == "all candidate states obtained a controller"
    assert list(o["iter_new_reachable"]) == [52481, 57431, 91549, 122322, 129220, 120161, 110237, 94948, 78464,
                                             64643, 43185, 16768]
    nc = list(o["iter_new_certified"])
    assert nc[:5] == [123510, 1097, 1502, 1501, 1459] and nc[7:] == [5579, 7315, 7976, 3937, 130]
    assert sha(o["reachable_mask"])[:16] == "086f49c353a25f80"
    assert sha(o["controller"])[:16] == "c1fbf29d702e1d9b"
    assert sha(o["reach_step"])[:16] == "276f76e476f846fa"


def test_prefix_and_query_match_direct_count():
    rng = np.random.default_rng(7)
    shape = (5, 4, 6, 3)
    mask = (rng.random(int(np.prod(shape))) < 0.4).astype(np.uint8)
    P = O.prefix(shape, mask)
    grid = mask.reshape(shape[::-1])   # [w][z][y][x]
    n0, n1, n2, n3 = shape
    for _ in range(200):
        lo = [int(rng.integers(0, n)) for n in shape]
        hi = [int(rng.integers(lo[d], shape[d])) for d in range(4)]
        wrap = rng.random() < 0.3 and lo[2] > 0
        if wrap:
            lo[2], hi[2] = hi[2], lo[2] - 1 if lo[2] > 0 else 0
            if lo[2] <= hi[2]:
                continue
        flat = lambda i: i[0] + n0 * (i[1] + n1 * (i[2] + n2 * i[3]))
        got = O.lib().orc_query((O.ctypes.c_uint32 * 4)(*shape), 2, O._ptr(P), flat(lo), flat(hi))
        zs = list(range(lo[2], hi[2] + 1)) if lo[2] <= hi[2] else list(range(lo[2], n2)) + list(range(0, hi[2] + 1))
        want = int(grid[lo[3]:hi[3] + 1][:, zs][:, :, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1].sum())
        assert got == want


def test_spot_step_agrees_with_full_solve():
    case = INDEX["hyperbolic_mid_a"]["case"]
    c1 = dict(case, max_iterations=3)
    c2 = dict(case, max_iterations=4)
    a = O.solve(c1)
    b = O.solve(c2)
    assert b["iterations"] == 4
    states = np.arange(a["states"], dtype=np.uint64)
    rn, ct, st = O.spot_step(case, a["valid_mask"], a["candidate_mask"], a["reachable_mask"], a["controller"],
                             a["reach_step"], 4, states)
    assert np.array_equal(rn, b["reachable_mask"])
    assert np.array_equal(ct, b["controller"])
    assert np.array_equal(st, b["reach_step"])


def test_simulation_oracle_matches_reference_fixtures():
    """oracle/sim_oracle.py against trajectories made by the reference's own
    get_control_input / update_state (tests/golden/make_sim_golden.py)."""
    import json
    import os

    import sim_oracle as S

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with open(os.path.join(here, "sim_index.json")) as f:
        sims = json.load(f)
    index = golden_index()
    for name in sims:
        case = index[name]["case"]
        z = np.load(os.path.join(here, f"sim_{name}.npz"))
        shape, ishape = C.grid_shape(case)
        grid = {"state_lb": case["state_lb"], "state_eta": case["state_eta"], "shape": list(shape),
                "input_lb": case["input_lb"], "input_eta": case["input_eta"], "input_shape": list(ishape),
                "sample_time": case["sample_time"], "integration_substeps": case["integration_substeps"],
                "disturbance_half_width": case["disturbance_half_width"]}
        traj, done = S.simulate(golden_arrays(name)["controller"], grid, z["x0"], int(z["steps"]), int(z["seed"]))
        assert np.array_equal(done, z["steps_done"]), name
        assert np.array_equal(traj, z["trajectories"]), name
        assert done.max() > 0 and done.min() == 0   # both stopped and running trajectories are covered

