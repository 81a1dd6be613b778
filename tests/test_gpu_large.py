"""Parity at the largest sizes, where the full CPU oracle is too slow:
  * 128x128x72x48 states x 144 inputs (8.2 G pairs): after the GPU's
    iteration k-1 (a solve capped at k-1 iterations), the oracle recomputes
    iteration k for 10^5 seeded states plus every state the GPU changed in
    iteration k (up to a cap), and must agree bit for bit with the GPU's
    solve capped at k iterations;
  * the fused method's widest rows (256 x-cells, 8 words) and grids wider
    than that or than 255 cells in any dimension (the stored method with
    16-bit box bounds), against the full oracle."""
import numpy as np
import pytest

import gsc_b200 as G
import gsc_cases as C
import oracle as O
from helpers import assert_same_result

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def capped(ctx, absn, case, k):
    q = C.clone(case, max_iterations=k)
    p = G.Problem(ctx, absn, q, G.METHOD_FUSED)
    p.solve(graph=True)
    r = p.read()
    p.close()
    return r


@pytest.mark.timeout(600)
def test_large_workload_spot_checked_per_iteration(ctx):
    case = C.large_case()
    absn = G.Abstraction(ctx, case)
    full = capped(ctx, absn, case, case["max_iterations"])
    assert full["iterations"] == 75 and full["message"] == "iteration stalled before candidate closure"
    rng = np.random.default_rng(11)
    S = full["states"]
    for k in (1, 2, 20, 75):
        a = capped(ctx, absn, case, k - 1)
        b = capped(ctx, absn, case, k)
        changed = np.flatnonzero((a["reachable_mask"] != b["reachable_mask"]) | (a["controller"] != b["controller"]))
        states = np.unique(np.concatenate([rng.integers(0, S, 100_000, dtype=np.uint64),
                                           changed[:50_000].astype(np.uint64)]))
        rn, ct, st = O.spot_step(case, a["valid_mask"], a["candidate_mask"], a["reachable_mask"], a["controller"],
                                 a["reach_step"], k, states)
        assert np.array_equal(rn, b["reachable_mask"][states]), k
        assert np.array_equal(ct, b["controller"][states]), k
        assert np.array_equal(st, b["reach_step"][states]), k
        if k < 75:
            assert changed.size > 0, k
    absn.close()


@pytest.mark.timeout(900)
def test_large_workload_stored_equals_fused(ctx):
    """128x128x72x48 x 144 with both methods side by side: the stored
    method's 65 GB of one-byte boxes (8 B per pair) streamed every iteration,
    against the fused method's recomputed boxes, bit for bit over the whole
    75-iteration fixpoint (the fused solve is spot-checked against the oracle
    above)."""
    case = C.large_case()
    absn = G.Abstraction(ctx, case)
    out = {}
    for method in (G.METHOD_FUSED, G.METHOD_STORED):
        p = G.Problem(ctx, absn, case, method)
        p.solve(graph=True)
        out[method] = p.read()
        assert p.timings()["method"] == method
        p.close()
        ctx.trim()
    assert_same_result(out[G.METHOD_STORED], out[G.METHOD_FUSED], "128x128x72x48 stored vs fused")
    assert out[G.METHOD_STORED]["iterations"] == out[G.METHOD_FUSED]["iterations"] == 75
    absn.close()


def test_widest_fused_rows(ctx):
    """256 x-cells: eight 32-bit words per row, the fused method's limit."""
    case = C.unicycle_grid_case((256, 16, 8, 6), (3, 3), "wide_256", max_iterations=64)
    want = O.solve(case)
    absn = G.Abstraction(ctx, case)
    p = G.Problem(ctx, absn, case, G.METHOD_AUTO)
    p.solve(graph=True)
    got = p.read()
    assert p.timings()["method"] == G.METHOD_FUSED
    p.close()
    assert_same_result(got, want, "nx=256")
    assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
    absn.close()


def wide_demo_case(n):
    """The published demo's geometry and dynamics on an n-cell grid, 5x5 inputs."""
    c = dict(C.hyperbolic_demo_case())
    c["name"] = "wide_demo_%dx%dx%dx%d" % tuple(n)
    c["state_eta"] = [(c["state_ub"][d] - c["state_lb"][d]) / n[d] for d in range(4)]
    c["input_eta"] = [0.4, 0.4]
    c["expect_shape"] = list(n)
    return C.checked(c)


@pytest.mark.parametrize("shape,demo", [((257, 16, 8, 6), False), ((300, 12, 10, 6), False),
                                        ((40, 300, 6, 4), False), ((300, 24, 20, 8), True)])
def test_wide_grids_take_the_stored_method_with_16_bit_bounds(ctx, shape, demo):
    """More than 256 x-cells is wider than the fused rows, and more than 255
    cells in any dimension wider than one-byte box bounds: the automatic
    choice is the stored method with 16-bit bounds, and the result is the
    oracle's bit for bit (the reference takes any grid of 32-bit state
    indices, grid.hpp:135).  The demo-geometry grid runs 52 iterations."""
    if demo:
        case = wide_demo_case(shape)
    else:
        case = C.unicycle_grid_case(shape, (3, 3), "wide_%dx%dx%dx%d" % shape, max_iterations=64)
    want = O.solve(case)
    absn = G.Abstraction(ctx, case)
    # The automatic choice: stored beyond the fused rows' 256 x-cells, else
    # fused (whose y, theta and v tables are 16-bit); then the stored method
    # with 16-bit bounds explicitly, from one CUDA graph and from the host loop.
    auto = G.METHOD_STORED if shape[0] > 256 else G.METHOD_FUSED
    for method, graph in ((G.METHOD_AUTO, True), (G.METHOD_STORED, True), (G.METHOD_STORED, False)):
        p = G.Problem(ctx, absn, case, method)
        p.solve(graph=graph)
        got = p.read()
        assert p.timings()["method"] == (auto if method == G.METHOD_AUTO else method)
        p.close()
        assert_same_result(got, want, "x".join(map(str, shape)) + f" method {method} graph {graph}")
        assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
        assert list(got["iter_new_reachable"]) == list(want["iter_new_reachable"])
    if shape[0] > 256:
        with pytest.raises(G.GscError) as e:
            G.Problem(ctx, absn, case, G.METHOD_FUSED)
        assert e.value.status == 4
    absn.close()


def test_boxes_wider_than_a_word_fall_back_to_stored(ctx):
    """x-boxes of more than 32 cells (a large x disturbance on 255 x-cells):
    the fused method refuses them, the automatic choice is the stored
    method, and the result is the oracle's."""
    case = C.unicycle_grid_case((255, 8, 6, 4), (3, 3), "wide_boxes", max_iterations=64)
    case["disturbance_half_width"] = [2.6, 0.01, 0.01, 0.01]
    want = O.solve(case)
    absn = G.Abstraction(ctx, case)
    p = G.Problem(ctx, absn, case, G.METHOD_AUTO)
    p.solve(graph=True)
    got = p.read()
    assert p.timings()["method"] == G.METHOD_STORED
    p.close()
    assert_same_result(got, want, "wide boxes")
    assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
    with pytest.raises(G.GscError) as e:
        G.Problem(ctx, absn, case, G.METHOD_FUSED)
    assert e.value.status == 4
    absn.close()
