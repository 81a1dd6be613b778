"""The sharded fixpoint on the device (gsc_problem_shard_*), ranks as threads.

Each rank is a thread with its own context (stream), abstraction and
problem on cuda:0, iterating its own contiguous slice range; the ranks
exchange their D' slabs and summed counts every iteration through
gsc_shard.ThreadComm (device copies), as processes on separate GPUs do
through NCCL.  No kernel waits on another: every exchange is a host-side
barrier between launches.  The gathered result must equal the reference's
(golden fixtures) and the regular one-GPU solve bit for bit."""
import numpy as np
import pytest

import gsc_b200 as G
import gsc_cases as C
import gsc_shard
from helpers import ARRAYS, assert_same_result, golden_arrays, golden_index

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,world", [("small", 2), ("hyperbolic_mid_b", 2), ("hyperbolic_mid_b", 3),
                                        ("wraparound", 2), ("default_empty_candidate", 2), ("small_maxiter0", 2),
                                        ("mini_instance_1", 4)])
def test_sharded_solve_matches_the_reference(name, world):
    meta = golden_index()[name]
    got = gsc_shard.solve_threads(meta["case"], world)
    want = golden_arrays(name)
    assert_same_result(got, {k: want[k] for k in ARRAYS}, f"{name} x{world}")
    assert got["iterations"] == meta["iterations"] and got["message"] == meta["message"]
    assert got["reachable_states"] == int(want["reachable_mask"].sum())


def test_sharded_demo_scale_matches_one_gpu_solve():
    """65x65x38x25 states x 100 inputs over two ranks, against the graph solve."""
    case = C.demo_scale_case()
    got = gsc_shard.solve_threads(case, 2)
    one = G.run_case(case, method=G.METHOD_FUSED, graph=True)
    assert_same_result(got, one, "demo_scale x2")
    assert got["iterations"] == one["iterations"] == 32 and got["message"] == one["message"]
    assert list(np.asarray(got["iter_new_reachable"][:32])) == list(np.asarray(one["iter_new_reachable"][:32]))


def test_a_regular_solve_after_a_sharded_one_covers_the_whole_grid():
    name = "hyperbolic_mid_a"
    case = golden_index()[name]["case"]
    ctx = G.Context(0)
    absn = G.Abstraction(ctx, case)
    p = G.Problem(ctx, absn, case, G.METHOD_FUSED)
    eng = gsc_shard.DeviceEngine(p)
    eng.begin(0, eng.slices // 2)
    eng.step()
    p.solve(graph=True)
    got = p.read()
    want = golden_arrays(name)
    assert_same_result(got, {k: want[k] for k in ARRAYS}, name)
    p.close()
    absn.close()
    ctx.close()
