"""Batched instances (gsc_batch_*): every instance of a batch gives exactly
the result of its own one-problem solve and of the reference CPU method --
masks, controller, reach_step, iteration count, stop message, per-iteration
counts -- whatever else shares the launches with it."""
import numpy as np
import pytest

import gsc_b200 as G
import gsc_cases as C
import oracle as O
from helpers import assert_same_result, golden_arrays, golden_index

pytestmark = pytest.mark.gpu
INDEX = golden_index()


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def solo(ctx, case):
    a = G.Abstraction(ctx, case)
    p = G.Problem(ctx, a, case, G.METHOD_FUSED)
    p.solve(graph=True)
    out = p.read()
    p.close()
    a.close()
    return out


def check_entry(got, name):
    entry = INDEX[name]
    assert_same_result(got, golden_arrays(name), f"batch/{name}")
    assert got["iterations"] == entry["iterations"], name
    assert got["converged"] == entry["converged"], name
    assert got["message"] == entry["message"], name
    assert got["reachable_states"] == entry["reachable_states"], name
    assert got["certified_candidates"] == entry["certified_candidates"], name


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "hostloop"])
def test_batch_of_golden_cases(ctx, graph):
    """All golden cases (different grids, inputs, obstacles, wrap-around,
    an empty candidate set, max_iterations 0) in one batch, read one by one
    and all at once."""
    names = sorted(INDEX)
    b = G.Batch(ctx, [INDEX[n]["case"] for n in names])
    b.solve(graph=graph)
    for i, n in enumerate(names):
        check_entry(b.read(i), n)
    for n, got in zip(names, b.read_all()):
        check_entry(got, n)
    rep = b.report()
    assert rep["instances"] == len(names)
    assert rep["max_iterations_run"] == max(INDEX[n]["iterations"] for n in names)
    assert rep["kernel_launches"] >= 1 + 4 * rep["max_iterations_run"] if graph else rep["kernel_launches"] > 0
    b.close()


def test_batch_random_instances_against_oracle(ctx):
    cases = [C.random_instance(4242, i, n_lo=(8, 8, 8, 6), n_hi=(28, 28, 20, 14)) for i in range(5)]
    b = G.Batch(ctx, cases)
    b.solve(graph=True)
    for i, c in enumerate(cases):
        got = b.read(i)
        want = O.solve(c)
        assert_same_result(got, want, f"instance {i}")
        assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
    b.close()


def test_batch_mixed_sizes_autotuned_match_solo(ctx):
    """Instances of the batched workload's full size range (one and two
    words per row), with different iteration caps, autotuned shapes, solved
    twice through the same graph."""
    cases = [C.random_instance(20261203, i) for i in range(4)]
    cases.append(C.clone(cases[0], max_iterations=0))
    cases.append(C.clone(cases[1], max_iterations=1))
    assert {(C.grid_shape(c)[0][0] + 31) // 32 for c in cases} >= {2}
    b = G.Batch(ctx, cases, autotune=True)
    rep = b.report()
    assert rep["tuned"] in (1, 2) and rep["sat_threads"] in (64, 128, 256)
    for rnd in range(2):
        b.solve(graph=True)
        for i, c in enumerate(cases):
            assert_same_result(b.read(i), solo(ctx, c), f"round {rnd} instance {i}")
    b.close()


@pytest.mark.parametrize("shape", [(64, 0, 1024, 0), (256, 4, 4096, 0), (128, 16, 256, 0), (128, 0, 1024, 1),
                                   (256, 8, 2048, 1)])
def test_batch_launch_shapes_agree(ctx, shape):
    """Block- and warp-per-task satisfaction launches, one block per task or
    persistent, give the golden results."""
    cases = [INDEX[n]["case"] for n in ("small_obstacles", "hyperbolic_mid_a", "wraparound", "mini_instance_2")]
    b = G.Batch(ctx, cases, sat_threads=shape[0], sat_blocks_per_sm=shape[1], chunk_words=shape[2],
                sat_warp_tasks=bool(shape[3]))
    assert b.report()["sat_warp_tasks"] == shape[3]
    b.solve(graph=bool(shape[1] % 8))
    for i, n in enumerate(("small_obstacles", "hyperbolic_mid_a", "wraparound", "mini_instance_2")):
        check_entry(b.read(i), n)
    b.close()


def test_batch_rejects_instance_outside_fused_method(ctx):
    ok = INDEX["small"]["case"]
    wide = C.unicycle_grid_case((300, 8, 8, 6), (3, 3))
    with pytest.raises(G.GscError) as e:
        G.Batch(ctx, [ok, wide])
    assert e.value.status == 4 and "instance 1" in str(e.value)
    # the context stays usable
    check_entry(solo(ctx, ok), "small")


def test_batch_rejects_bad_options(ctx):
    with pytest.raises(G.GscError) as e:
        G.Batch(ctx, [INDEX["small"]["case"]], sat_threads=96)
    assert e.value.status == 1


def test_batch_with_instances_that_fill_the_gpu(ctx):
    """Instances of 65x65x38x25 states x 100 inputs (4 x 10^8 pairs) iterate
    with the one-problem kernels inside the batch, the small ones with the
    batched kernels; every result is its solo solve's, in the graph (launch
    shapes autotuned) and the host loop.  Without autotuning (which iterates
    the small instances to time them), a report before the first solve reads
    no iterations from the recycled pool memory."""
    demo = C.demo_scale_case()
    cases = [demo, INDEX["small_obstacles"]["case"], C.clone(demo, max_iterations=5), INDEX["hyperbolic_mid_a"]["case"]]
    want = [solo(ctx, c) for c in cases]
    for graph in (True, False):
        b = G.Batch(ctx, cases, autotune=graph)
        if not graph:
            assert b.report()["max_iterations_run"] == 0
        b.solve(graph=graph)
        for i, got in enumerate(b.read_all()):
            assert_same_result(got, want[i], f"graph={graph} instance {i}")
            assert got["iterations"] == want[i]["iterations"] and got["message"] == want[i]["message"]
        assert b.report()["max_iterations_run"] == max(w["iterations"] for w in want)
        b.close()


@pytest.mark.parametrize("part", [1, 3, 0, 100])
def test_batch_run_pipelined_matches_golden_and_solo(ctx, part):
    """gsc_batch_run: parts that overlap set-up, solve and copies give every
    instance its golden (reference) result or its solo solve, whatever the
    part size (one instance a part, uneven parts, the default, one part)."""
    names = sorted(INDEX)
    cases = [INDEX[n]["case"] for n in names] + [C.random_instance(777, i) for i in range(3)]
    got = G.run_batch(ctx, cases, autotune=(part == 3), part_instances=part)
    for i, n in enumerate(names):
        check_entry(got[i], n)
    for i, c in enumerate(cases[len(names):], start=len(names)):
        want = solo(ctx, c)
        assert_same_result(got[i], want, f"part={part} instance {i}")
        assert got[i]["iterations"] == want["iterations"] and got[i]["message"] == want["message"]


def test_batch_run_reports_the_failing_part(ctx):
    ok = INDEX["small"]["case"]
    wide = C.unicycle_grid_case((300, 8, 8, 6), (3, 3))
    with pytest.raises(G.GscError) as e:
        G.run_batch(ctx, [ok, ok, wide, ok], part_instances=2)
    assert e.value.status == 4 and "instances 2..3" in str(e.value)
    check_entry(solo(ctx, ok), "small")
