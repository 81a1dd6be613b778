"""The serving loop (gsc_server_*): queries against resident abstractions,
admitted by a memory budget and iterated together as they arrive.  Each
served result must be bit-identical to the same query solved alone, and to
the reference CPU method where that is cheap."""
import time

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


@pytest.fixture(scope="module")
def models(ctx):
    cases = {"small": C.small_case(), "mid": C.serve_mid_case(),
             "tiny": C.unicycle_grid_case((12, 14, 10, 8), (4, 5), "tiny")}
    absn = {k: G.Abstraction(ctx, c) for k, c in cases.items()}
    yield cases, absn
    for a in absn.values():
        a.close()


def alone(ctx, abs_, q):
    p = G.Problem(ctx, abs_, q, G.METHOD_FUSED)
    p.solve(graph=True)
    out = p.read()
    p.close()
    return out


@pytest.mark.parametrize("warp", [False, True], ids=["block_tasks", "warp_tasks"])
def test_served_mix_matches_alone(ctx, models, warp):
    cases, absn = models
    srv = G.Server(ctx, memory_budget=2 << 30, iterations_per_step=1, sat_warp_tasks=warp)
    queries = []
    for i in range(36):
        k = ("small", "mid", "tiny")[i % 3]
        queries.append((k, C.random_query(cases[k], 11, i)))
    tickets = [srv.submit(absn[k], q) for k, q in queries]
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(queries) and st["failed"] == 0
    assert st["max_running"] > 1, "queries never iterated together"
    assert st["peak_device_bytes"] <= st["device_bytes_budget"]
    for (k, q), got in zip(queries, results):
        assert got["status"] == 0 and got["latency_ms"] > 0
        want = alone(ctx, absn[k], q)
        assert_same_result(got, want, q["name"])
        for f in ("iterations", "message", "converged", "reachable_states", "certified_candidates"):
            assert got[f] == want[f], (q["name"], f)


def test_served_against_oracle(ctx, models):
    cases, absn = models
    srv = G.Server(ctx, memory_budget=1 << 30)
    qs = [C.random_query(cases["tiny"], 5, i, iter_lo=1, iter_hi=40) for i in range(4)]
    tickets = [srv.submit(absn["tiny"], q) for q in qs]
    for q, t in zip(qs, tickets):
        got = srv.wait(t)
        want = O.solve(q)
        assert_same_result(got, want, q["name"])
        assert got["iterations"] == want["iterations"] and got["message"] == want["message"]
    srv.close()


def test_budget_admission_queues_and_completes(ctx, models):
    """A budget that holds only a few queries at once: the rest wait for
    memory, every query completes with the same result as alone, and the
    pool never exceeds the budget."""
    cases, absn = models
    one = alone(ctx, absn["mid"], C.random_query(cases["mid"], 3, 0))
    srv = G.Server(ctx, memory_budget=48 << 20, max_slots=64)
    qs = [C.random_query(cases["mid"], 3, i) for i in range(10)]
    tickets = [srv.submit(absn["mid"], q) for q in qs]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == 10 and st["failed"] == 0
    assert st["peak_device_bytes"] <= st["device_bytes_budget"] <= 48 << 20
    assert st["max_running"] < 10
    assert_same_result(res[0], one, "first query")
    for q, got in zip(qs[1:4], res[1:4]):
        assert_same_result(got, alone(ctx, absn["mid"], q), q["name"])


def test_failures_stay_with_their_query(ctx, models):
    cases, absn = models
    srv = G.Server(ctx, memory_budget=8 << 20)
    good = C.random_query(cases["tiny"], 9, 0)
    bad_cand = C.clone(good, candidate="rect", candidate_lb=[-2, -2, -4, 0], candidate_ub=[2, 2, 4, 1],
                       obstacles=[[-0.5, -0.5, -4, 0, 0.5, 0.5, 4, 1]])
    too_big = C.random_query(cases["mid"], 9, 1)   # does not fit 8 MiB
    zero = C.clone(good, max_iterations=0)
    t = [srv.submit(absn["tiny"], good), srv.submit(absn["tiny"], bad_cand), srv.submit(absn["mid"], too_big),
         srv.submit(absn["tiny"], zero)]
    r0 = srv.wait(t[0])
    r1 = srv.wait(t[1], check=False)
    r2 = srv.wait(t[2], check=False)
    r3 = srv.wait(t[3])
    srv.close()
    assert r1["status"] == 6     # candidate set contains invalid states
    assert r2["status"] == 3     # out of device memory
    assert_same_result(r0, alone(ctx, absn["tiny"], good), "good")
    assert r3["iterations"] == 0 and r3["message"] == "maximum iterations reached"
    assert_same_result(r3, alone(ctx, absn["tiny"], zero), "zero")


def test_wait_timeout_and_unknown_ticket(ctx, models):
    cases, absn = models
    srv = G.Server(ctx, memory_budget=256 << 20)
    with pytest.raises(G.GscError) as e:
        srv.wait(12345, timeout_ms=0)
    assert e.value.status == 1
    t = srv.submit(absn["small"], C.random_query(cases["small"], 1, 0))
    deadline = time.time() + 60
    while True:
        try:
            srv.wait(t, timeout_ms=0)
            break
        except G.GscError as err:
            assert err.status == 7
            assert time.time() < deadline
            time.sleep(0.001)
    srv.close()


def test_served_queries_that_fill_the_gpu_match_alone(ctx, models):
    """Queries on a 65x65x38x25 x 100 grid (4 x 10^8 pairs) iterate with the
    one-problem kernels next to small queries on the batched kernels; each
    result is the same query's solved alone."""
    cases, absn = models
    demo = C.demo_scale_case()
    a_demo = G.Abstraction(ctx, demo)
    srv = G.Server(ctx, memory_budget=6 << 30, iterations_per_step=1)
    queries = []
    for i in range(12):
        k = ("demo", "small", "mid")[i % 3]
        queries.append((k, C.random_query(demo if k == "demo" else cases[k], 23, i)))
    abs_of = {"demo": a_demo, "small": absn["small"], "mid": absn["mid"]}
    tickets = [srv.submit(abs_of[k], q) for k, q in queries]
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(queries) and st["failed"] == 0
    assert st["max_running"] > 1
    for (k, q), got in zip(queries, results):
        assert got["status"] == 0
        want = alone(ctx, abs_of[k], q)
        assert_same_result(got, want, q["name"])
        for f in ("iterations", "message", "converged", "reachable_states", "certified_candidates"):
            assert got[f] == want[f], (q["name"], f)
    a_demo.close()
