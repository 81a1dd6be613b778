"""The allocation-free fixpoint (gsc_fixpoint_noalloc) against the regular path.

gsc_fixpoint_noalloc exists for callers that cannot call cudaMalloc when they
solve: they hold the abstraction and the output arrays in device memory they
already own, and the library's working tables live in a fixed device array.
This test builds an abstraction with the regular entry points, exports it in
the reference's layout, then calls gsc_fixpoint_noalloc twice in a row on the
same arrays (outputs overwritten with junk before each call) and requires the
regular path's results bit for bit both times.  The cases cover every way a
solve stops: convergence, a stall, the iteration cap, and a cap of zero; and
a theta-wrapped grid.  The file is collected last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import gsc_b200 as G
from helpers import golden_arrays, golden_index

pytestmark = pytest.mark.gpu


def _dev(torch, arr, device):
    a = np.ascontiguousarray(arr)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).to(device)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _regular(case):
    """The regular path's result and its exported abstraction."""
    ctx = G.Context(0)
    abs_ = G.Abstraction(ctx, case)
    prob = G.Problem(ctx, abs_, case, G.METHOD_AUTO)
    prob.solve(graph=True)
    want = prob.read()
    mn, mx, pv = prob.export_abstraction()
    prob.close()
    abs_.close()
    ctx.close()
    return want, mn, mx, pv


# (golden case, max_iterations override or None, the stop message expected)
CASES = [
    ("hyperbolic_mid_b", None, "iteration stalled before candidate closure"),   # 34 iterations
    ("default_empty_candidate", None, "all candidate states obtained a controller"),
    ("small_maxiter0", None, "maximum iterations reached"),                     # cap of zero
    ("hyperbolic_mid_b", 5, "maximum iterations reached"),                      # cap reached
    ("wraparound", None, "iteration stalled before candidate closure"),
    ("wraparound_full_circle", None, "iteration stalled before candidate closure"),
]


@pytest.mark.parametrize("name,cap,message", CASES, ids=[f"{c[0]}-cap{c[1]}" for c in CASES])
def test_noalloc_fixpoint_matches_regular_path_twice(name, cap, message):
    torch = pytest.importorskip("torch")
    case = dict(golden_index()[name]["case"])
    if cap is not None:
        case["max_iterations"] = cap
    want, mn, mx, pv = _regular(case)
    assert want["message"] == message
    if cap is None:
        ref = golden_arrays(name)
        assert np.array_equal(want["reachable_mask"], ref["reachable_mask"])

    dev = torch.device("cuda", 0)
    shape = (ctypes.c_uint32 * 4)(*want["shape"])
    d_mn, d_mx, d_pv = _dev(torch, mn, dev), _dev(torch, mx, dev), _dev(torch, pv, dev)
    d_valid = _dev(torch, want["valid_mask"], dev)
    d_cand = _dev(torch, want["candidate_mask"], dev)
    S = want["states"]
    reach = torch.empty(S, dtype=torch.uint8, device=dev)
    ctl = torch.empty(S, dtype=torch.int32, device=dev)
    step = torch.empty(S, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        reach.fill_(7 + call)
        ctl.fill_(12345)
        step.fill_(-3)
        summary = G.Result()
        st = G.lib().gsc_fixpoint_noalloc(shape, want["inputs"], 2, _ptr(d_mn), _ptr(d_mx), _ptr(d_pv),
                                          _ptr(d_valid), _ptr(d_cand), case["max_iterations"], _ptr(reach),
                                          _ptr(ctl), _ptr(step), ctypes.byref(summary), ctypes.c_void_p(stream))
        assert st == 0, G.STATUS.get(st, st)
        torch.cuda.synchronize(dev)
        assert np.array_equal(reach.cpu().numpy(), want["reachable_mask"]), f"call {call}: reachable_mask"
        assert np.array_equal(ctl.cpu().numpy().view(np.uint32), want["controller"]), f"call {call}: controller"
        assert np.array_equal(step.cpu().numpy().view(np.uint32), want["reach_step"]), f"call {call}: reach_step"
        assert summary.iterations == want["iterations"]
        assert G.MESSAGES[summary.message] == want["message"]
        assert summary.reachable_states == want["reachable_states"]
        assert summary.certified_candidates == want["certified_candidates"]
        assert summary.candidate_count == want["candidate_count"]


def test_noalloc_refuses_candidates_outside_the_valid_set():
    """abstraction.hpp:268-272: a candidate set with an invalid state is an error."""
    torch = pytest.importorskip("torch")
    name = "small"
    case = golden_index()[name]["case"]
    want, mn, mx, pv = _regular(case)
    dev = torch.device("cuda", 0)
    shape = (ctypes.c_uint32 * 4)(*want["shape"])
    d_mn, d_mx, d_pv = _dev(torch, mn, dev), _dev(torch, mx, dev), _dev(torch, pv, dev)
    d_valid = _dev(torch, want["valid_mask"], dev)
    cand = want["candidate_mask"].copy()
    bad = int(np.flatnonzero(want["valid_mask"] == 0)[0])
    cand[bad] = 1
    d_cand = _dev(torch, cand, dev)
    S = want["states"]
    reach = torch.empty(S, dtype=torch.uint8, device=dev)
    ctl = torch.empty(S, dtype=torch.int32, device=dev)
    step = torch.empty(S, dtype=torch.int32, device=dev)
    st = G.lib().gsc_fixpoint_noalloc(shape, want["inputs"], 2, _ptr(d_mn), _ptr(d_mx), _ptr(d_pv), _ptr(d_valid),
                                      _ptr(d_cand), case["max_iterations"], _ptr(reach), _ptr(ctl), _ptr(step), None,
                                      None)
    assert st == 6   # GSC_ERR_CANDIDATE_INVALID


def test_noalloc_refuses_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.int32, device=dev)
    p = _ptr(buf)
    too_big = (ctypes.c_uint32 * 4)(128, 128, 72, 48)   # 59.5 M padded entries
    st = G.lib().gsc_fixpoint_noalloc(too_big, 144, 2, p, p, p, p, p, 10, p, p, p, None, None)
    assert st == 3   # GSC_ERR_OUT_OF_MEMORY, before any device work
    # 16^4 states: a max_iterations argument of min(100000, 65537), beyond the 4,094 the scratch counts.
    many_iters = (ctypes.c_uint32 * 4)(16, 16, 16, 16)
    st = G.lib().gsc_fixpoint_noalloc(many_iters, 4, 2, p, p, p, p, p, 100000, p, p, p, None, None)
    assert st == 3   # refused before any device work
