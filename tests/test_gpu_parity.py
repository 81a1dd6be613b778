"""Parity of the CUDA path (through the C ABI) with the reference CPU method:
bit-exact masks, controller, reach_step, iteration count, stop message and
per-iteration counts, for both methods, host-driven and graph-driven loops."""
import hashlib

import numpy as np
import pytest

import gsc_b200 as G
import gsc_cases as C
import oracle as O
from helpers import assert_same_result, golden_arrays, golden_index

pytestmark = pytest.mark.gpu
INDEX = golden_index()
METHODS = {"stored": G.METHOD_STORED, "fused": G.METHOD_FUSED}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def solve(ctx, case, method, graph, **masks):
    a = G.Abstraction(ctx, case)
    p = G.Problem(ctx, a, case, method, **masks)
    p.solve(graph=graph)
    out = p.read()
    out["timings"] = p.timings()
    p.close()
    a.close()
    return out


@pytest.mark.parametrize("graph", [False, True], ids=["hostloop", "graph"])
@pytest.mark.parametrize("method", sorted(METHODS))
@pytest.mark.parametrize("name", sorted(INDEX))
def test_golden_parity(ctx, name, method, graph):
    entry = INDEX[name]
    got = solve(ctx, entry["case"], METHODS[method], graph)
    assert got["timings"]["method"] == METHODS[method]
    assert_same_result(got, golden_arrays(name), f"{name}/{method}")
    assert got["iterations"] == entry["iterations"]
    assert got["converged"] == entry["converged"]
    assert got["message"] == entry["message"]
    assert got["reachable_states"] == entry["reachable_states"]
    assert got["certified_candidates"] == entry["certified_candidates"]


@pytest.mark.parametrize("name", sorted(INDEX))
def test_abstraction_export_matches_reference(ctx, name):
    entry = INDEX[name]
    if "abstraction_sha256" not in entry:
        pytest.skip("no abstraction digest")
    case = entry["case"]
    a = G.Abstraction(ctx, case)
    p = G.Problem(ctx, a, case, G.METHOD_AUTO)
    mn, mx, v = p.export_abstraction()
    assert sha(v) == entry["abstraction_sha256"]["valid"]
    assert sha(mn) == entry["abstraction_sha256"]["min_flat"]
    assert sha(mx) == entry["abstraction_sha256"]["max_flat"]


def test_run_case_one_shot(ctx):
    entry = INDEX["hyperbolic_mid_b"]
    got = G.run_case(entry["case"])
    assert_same_result(got, golden_arrays("hyperbolic_mid_b"), "run_case")
    assert got["iterations"] == entry["iterations"]


@pytest.mark.parametrize("method", sorted(METHODS))
def test_published_demo(ctx, method):
    """examples/hyperbolic_case.cfg against README.md:44-98 and the reference
    CPU outputs' digests."""
    o = solve(ctx, C.hyperbolic_demo_case(), METHODS[method], graph=True)
    assert o["reachable_states"] == 1142689 and o["certified_candidates"] == 161280
    assert o["iterations"] == 12 and o["converged"]
    assert list(o["iter_new_reachable"]) == [52481, 57431, 91549, 122322, 129220, 120161, 110237, 94948, 78464,
                                             64643, 43185, 16768]
    assert sha(o["reachable_mask"])[:16] == "086f49c353a25f80"
    assert sha(o["controller"])[:16] == "c1fbf29d702e1d9b"
    assert sha(o["reach_step"])[:16] == "276f76e476f846fa"


@pytest.mark.parametrize("method", sorted(METHODS))
def test_demo_scale_against_oracle_digests(ctx, method):
    """65x65x38x25 x 100 inputs: 32 iterations; digests from the oracle, which
    the reference CPU run reproduces."""
    o = solve(ctx, C.demo_scale_case(), METHODS[method], graph=True)
    assert o["iterations"] == 32 and o["reachable_states"] == 448560 and o["certified_candidates"] == 343856
    assert o["message"] == "iteration stalled before candidate closure"
    assert sha(o["reachable_mask"])[:16] == "300b474546565191"
    assert sha(o["controller"])[:16] == "9194b475f386eef1"
    assert sha(o["reach_step"])[:16] == "87b248e6afdafcb8"


@pytest.mark.parametrize("index", range(3))
def test_random_instances_against_oracle(ctx, index):
    case = C.random_instance(777, index, n_lo=(8, 8, 8, 6), n_hi=(28, 28, 20, 14))
    want = O.solve(case)
    for method in METHODS.values():
        got = solve(ctx, case, method, graph=bool(index % 2))
        assert_same_result(got, want, f"instance{index}/{method}")
        assert got["iterations"] == want["iterations"] and got["message"] == want["message"]


def demo_variant(i):
    """The published demo's geometry and dynamics on a seeded grid (20–72 x
    20–72 x 16–48 x 5–12 cells), input steps and substep count: fixpoints of
    6 to 44 iterations on rows of one to three words."""
    rng = np.random.default_rng([4242, i])
    c = dict(C.hyperbolic_demo_case())
    n = [int(rng.integers(20, 73)), int(rng.integers(20, 73)), int(rng.integers(16, 49)), int(rng.integers(5, 13))]
    c["name"] = "demo_variant_%d" % i
    c["state_eta"] = [(c["state_ub"][d] - c["state_lb"][d]) / n[d] for d in range(4)]
    c["input_eta"] = [float(rng.choice([0.4, 0.5, 2.0 / 3.0])), float(rng.choice([0.4, 0.5, 2.0 / 3.0]))]
    c["integration_substeps"] = int(rng.choice([4, 8, 16]))
    c["expect_shape"] = n
    return C.checked(c)


@pytest.mark.parametrize("index", range(8))
def test_demo_variants_against_oracle(ctx, index):
    """Deep fixpoints on odd grid shapes (incremental iterations, row-lost
    tests, several words per row) through both methods and both loops."""
    case = demo_variant(index)
    want = O.solve(case)
    for method in METHODS.values():
        for graph in (False, True):
            got = solve(ctx, case, method, graph)
            assert_same_result(got, want, f"{case['name']}/{method}/graph={graph}")
            assert got["iterations"] == want["iterations"] and got["message"] == want["message"]


@pytest.mark.parametrize("shape", [(1, 9, 8, 3), (9, 1, 8, 3), (33, 5, 1, 3), (17, 6, 8, 1), (1, 1, 1, 1),
                                   (32, 32, 2, 2), (64, 33, 3, 2)])
def test_degenerate_grids_against_oracle(ctx, shape):
    """Grids of one cell along a dimension (one theta cell: every box wraps
    the whole circle), one-cell grids and rows of exactly one or two words:
    each method that takes the grid gives the oracle's result."""
    c = dict(C.hyperbolic_demo_case())
    c["name"] = "degenerate_%dx%dx%dx%d" % shape
    c["state_eta"] = [(c["state_ub"][d] - c["state_lb"][d]) / shape[d] for d in range(4)]
    c["input_eta"] = [2.0 / 3.0, 2.0 / 3.0]
    c["integration_substeps"] = 4
    c["expect_shape"] = list(shape)
    case = C.checked(c)
    want = O.solve(case)
    solved = 0
    for method in (G.METHOD_AUTO, G.METHOD_STORED, G.METHOD_FUSED):
        for graph in (False, True):
            try:
                got = solve(ctx, case, method, graph)
            except G.GscError as e:
                assert method == G.METHOD_FUSED and e.status == 4, e   # fused refuses: stored takes it
                continue
            assert_same_result(got, want, f"{c['name']}/{method}/graph={graph}")
            assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
            solved += 1
    assert solved >= 4


def test_safe_mask_overrides(ctx):
    """A custom constraint (ConstraintType::kCustom) arrives as a host mask:
    rank 2 over (x, y) and rank 4 over all cells give the oracle's result."""
    case = INDEX["small_obstacles"]["case"]
    want = golden_arrays("small_obstacles")
    shape, _ = O.shapes(case)
    S = int(np.prod(shape))
    # rank 4: safe at every centre, evaluated by the oracle's valid mask with no map/obstacles
    free = dict(case, obstacles=[], map_lb=[-9, -9, -9, -9], map_ub=[9, 9, 9, 9], candidate="rect",
                candidate_lb=[9, 9, 9, 9], candidate_ub=[9, 9, 9, 9])
    safe4, _ = O.masks(free)
    safe2 = safe4[: shape[0] * shape[1]].copy()
    custom = dict(case, constraint="none")   # the mask alone carries the constraint (kCustom route)
    for rank, mask in ((2, safe2), (4, safe4)):
        for method in METHODS.values():
            for c in (case, custom):
                got = solve(ctx, c, method, graph=False, safe_mask=mask, safe_rank=rank)
                assert_same_result(got, want, f"safe rank {rank}/{method}/{c['constraint']}")
    assert S == safe4.size


def test_candidate_not_valid_is_rejected(ctx):
    case = C.default_case()
    case["candidate_lb"] = [0.5, -0.5, -C.PI, 0.0]   # overlaps the obstacle
    case["candidate_ub"] = [1.0, 0.5, C.PI, 2.0]
    a = G.Abstraction(ctx, case)
    with pytest.raises(G.GscError) as e:
        G.Problem(ctx, a, case, G.METHOD_AUTO)
    assert e.value.status == 6


def test_resolve_same_problem_twice(ctx):
    case = INDEX["hyperbolic_mid_a"]["case"]
    a = G.Abstraction(ctx, case)
    for method in METHODS.values():
        p = G.Problem(ctx, a, case, method)
        p.solve(graph=True)
        r1 = p.read()
        p.solve(graph=True)
        r2 = p.read()
        p.solve(graph=False)
        r3 = p.read()
        assert_same_result(r1, golden_arrays("hyperbolic_mid_a"), "first")
        assert_same_result(r2, r1, "graph relaunch")
        assert_same_result(r3, r1, "host loop after graph")


@pytest.mark.parametrize("cap", [1, 2, 3, 5, 8, 13, 33, 34, 35])
def test_max_iterations_stop_against_oracle(ctx, cap):
    """A solve cut off by max_iterations (reachability.hpp:141-144) at every
    stage of hyperbolic_mid_b's 34 iterations: the host loop (which queues
    iterations ahead of the stop word) and the graph give the oracle's bits,
    iteration count and message, for both methods."""
    case = dict(INDEX["hyperbolic_mid_b"]["case"], max_iterations=cap)
    want = O.solve(case)
    assert want["iterations"] == min(cap, 34)
    for method in METHODS.values():
        for graph in (False, True):
            got = solve(ctx, case, method, graph)
            assert_same_result(got, want, f"cap {cap}/{method}/graph={graph}")
            assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
            assert got["converged"] == want["converged"]


def test_context_on_a_caller_stream():
    """A context bound to the caller's CUDA stream (a torch stream here): both
    loops run on it and give the fixture's result, for both methods."""
    torch = pytest.importorskip("torch")
    s = torch.cuda.Stream(device=0)
    name = "hyperbolic_mid_b"
    with G.Context(0, stream=s.cuda_stream) as c:
        for method in METHODS.values():
            for graph in (False, True):
                got = solve(c, INDEX[name]["case"], method, graph)
                assert_same_result(got, golden_arrays(name), f"caller stream {method} graph={graph}")
                assert got["iterations"] == INDEX[name]["iterations"]
    torch.cuda.synchronize(0)


def test_context_pool_reuse_budget_and_trim():
    """Problems of a context draw on its caching pool: a second create/destroy
    cycle needs no new device memory, trim returns every unused region, and a
    budget below an abstraction's needs is refused with GSC_ERR_OUT_OF_MEMORY."""
    case = INDEX["small"]["case"]
    with G.Context(0) as c:
        a = G.Abstraction(c, case)
        p = G.Problem(c, a, case, G.METHOD_FUSED)
        p.solve(graph=True)
        first = p.read()
        p.close()
        held = c.memory_in_use()
        assert held > 0
        for _ in range(3):
            p = G.Problem(c, a, case, G.METHOD_FUSED)
            p.solve(graph=True)
            assert_same_result(p.read(), first, "reuse")
            p.close()
        assert c.memory_in_use() == held
        a.close()
        c.trim()
        assert c.memory_in_use() == 0
        c.set_memory_budget(1 << 20)   # below the abstraction's 1.3 MB of tables
        with pytest.raises(G.GscError) as e:
            G.Abstraction(c, case)
        assert e.value.status == 3
        assert c.memory_in_use() <= 1 << 20
        c.set_memory_budget(0)
        got = solve(c, case, G.METHOD_FUSED, True)
        assert_same_result(got, first, "after budget")
