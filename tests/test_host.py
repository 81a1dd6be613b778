"""Host-side logic that needs no GPU: the C ABI library loads and exports every
symbol include/gsc_b200.h declares, grid shapes, case generators, and the
no-device error path (no CPU fallback)."""
import os
import re

import numpy as np
import pytest

import gsc_b200 as G
import gsc_cases as C
import oracle as O
from helpers import ROOT


def declared_functions():
    with open(os.path.join(ROOT, "include", "gsc_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*[\w\s\*]+?\b(gsc_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = G.lib()
    names = declared_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(G.SIGNATURES)


def test_backend_compiled_and_abi():
    assert G.cuda_backend_compiled()
    assert G.lib().gsc_abi_version() == 1
    assert G.lib().gsc_message_string(2) == b"iteration stalled before candidate closure"
    assert G.lib().gsc_status_string(6) == b"candidate set contains invalid states"


@pytest.mark.parametrize("name", sorted(C.PRESETS))
def test_grid_shape_matches_reference_rule(name):
    case = C.PRESETS[name]()
    assert G.grid_shape(case) == O.shapes(case)
    C.checked(case)


def test_grid_shape_rejects_bad_grid():
    case = C.default_case()
    case["state_eta"][0] = 0.0
    with pytest.raises(G.GscError):
        G.grid_shape(case)
    case = C.default_case()
    case["wrap_dim"] = 1
    with pytest.raises(G.GscError) as e:
        G.grid_shape(case)
    assert e.value.status == 4


def test_random_instance_is_deterministic_and_in_range():
    a = C.random_instance(20261203, 5)
    b = C.random_instance(20261203, 5)
    assert a == b
    s, u = C.grid_shape(a)
    assert all(16 <= s[d] <= hi for d, hi in enumerate((48, 48, 32, 24)))
    assert 25 <= u[0] * u[1] <= 100
    assert 0.05 <= a["sample_time"] <= 0.2
    assert 0.005 <= a["disturbance_half_width"][0] <= 0.02


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_device_fails_loudly():
    with pytest.raises(G.GscError) as e:
        G.Context(0)
    assert e.value.status == 5
    with pytest.raises(G.GscError):
        G.run_case(C.default_case())


def test_bench_reads_the_committed_kernel_figures():
    """bench.py's roofline takes the dominant kernel's DRAM traffic and warp
    instructions per launch from the committed ncu summaries; both are there
    for the default workload, and the issue roofline computes from them."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    workload = C.PRESETS["demo_scale"]()["name"]
    traffic = bench.ncu_traffic("k_sat_col", workload)
    assert traffic and 1e6 < traffic < 1e9
    issue = bench.issue_roofline("k_sat_col", workload, 0.03, 1965.0, 148)
    assert issue and 1e6 < issue["warp_instructions_per_launch"] < 1e9
    assert abs(issue["peak"] - 4 * 148 * 1.965e9 / 1e12) < 1e-9 and 0 < issue["frac"] < 1.5
    assert bench.issue_roofline("k_sat_col", "no_such_workload", 0.03, 1965.0, 148) is None
