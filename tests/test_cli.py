"""The gsc host API and CLI (gpu-inner-outer_b200/host): the .cfg parser reads
the same cases as the Python presets, and --gpu reproduces the reference's
results through run_case_cuda_u32."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import gsc_cases as C
from helpers import ROOT, golden_arrays, golden_index

CLI = os.path.join(ROOT, "gpu-inner-outer_b200", "gsc_b200_cli")
CFG = os.path.join(ROOT, "gpu-inner-outer_b200", "configs")


def parsed(name):
    out = subprocess.run([CLI, os.path.join(CFG, name), "--print-config"], check=True, capture_output=True,
                         text=True).stdout
    return json.loads(out)


@pytest.mark.parametrize("cfg,preset", [("hyperbolic_demo.cfg", "hyperbolic_demo"),
                                        ("unicycle_small.cfg", "small"),
                                        ("unicycle_demo_scale.cfg", "demo_scale"),
                                        ("unicycle_large.cfg", "large")])
def test_config_files_match_presets(cfg, preset):
    got = parsed(cfg)
    want = C.PRESETS[preset]()
    for k in ("state_lb", "state_ub", "state_eta", "input_lb", "input_ub", "input_eta", "map_lb", "map_ub",
              "disturbance_half_width"):
        assert got[k] == [float(v) for v in want[k]], k
    assert got["sample_time"] == want["sample_time"]
    assert got["integration_substeps"] == want["integration_substeps"]
    assert got["max_iterations"] == want["max_iterations"]
    if want["constraint"] == "quadric":
        assert got["constraint_type"] == 3 and got["quadric"] == [float(v) for v in want["constraint_params"]]
        assert got["candidate_shape"] == 1 and got["candidate_ellipse"] == [float(v) for v in want["candidate_ellipse"]]
    else:
        assert got["constraint_type"] == 1 and got["hyperbolic"] == [float(v) for v in want["constraint_params"][:3]]
        assert got["candidate_lb"] == want["candidate_lb"] and got["candidate_ub"] == want["candidate_ub"]


def test_parser_rejects_unknown_keys(tmp_path):
    p = tmp_path / "bad.cfg"
    p.write_text("name = x\nnot_a_key = 3\n")
    r = subprocess.run([CLI, str(p), "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown config key: not_a_key" in r.stderr
    p.write_text("state_lb = 1, 2, 3\n")
    r = subprocess.run([CLI, str(p), "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1 and "state_lb expects 4" in r.stderr


def test_cpu_mode_is_refused():
    r = subprocess.run([CLI, os.path.join(CFG, "hyperbolic_demo.cfg"), "--cpu"], capture_output=True, text=True)
    assert r.returncode == 2 and "CPU method" in r.stderr


@pytest.mark.gpu
def test_cli_compare_exit_code_contract():
    """--compare: the reference's exit codes over the two device methods."""
    r = subprocess.run([CLI, os.path.join(CFG, "unicycle_small.cfg"), "--compare"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "exact_match   : true" in r.stdout and "[stored]" in r.stdout and "[fused]" in r.stdout


def _read(d, name, dtype):
    return np.fromfile(os.path.join(d, name), dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["fused", "stored"])
def test_cli_gpu_reproduces_published_demo(tmp_path, method):
    d = str(tmp_path / "out")
    r = subprocess.run([CLI, os.path.join(CFG, "hyperbolic_demo.cfg"), "--gpu", "--method", method, "--output", d],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "reachable     : 1142689" in r.stdout and "iterations    : 12" in r.stdout
    assert "message       : all candidate states obtained a controller" in r.stdout
    h = lambda a: hashlib.sha256(a.tobytes()).hexdigest()[:16]
    assert h(_read(d, "reachable_mask.u8", np.uint8)) == "086f49c353a25f80"
    assert h(_read(d, "controller.u32", np.uint32)) == "c1fbf29d702e1d9b"
    assert h(_read(d, "reach_step.u32", np.uint32)) == "276f76e476f846fa"


@pytest.mark.gpu
def test_cli_gpu_small_matches_reference_golden(tmp_path):
    d = str(tmp_path / "out")
    r = subprocess.run([CLI, os.path.join(CFG, "unicycle_small.cfg"), "--gpu", "--output", d], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    want = golden_arrays("small")
    for name, dt, key in (("reachable_mask.u8", np.uint8, "reachable_mask"), ("controller.u32", np.uint32, "controller"),
                          ("reach_step.u32", np.uint32, "reach_step"), ("valid_mask.u8", np.uint8, "valid_mask"),
                          ("candidate_mask.u8", np.uint8, "candidate_mask")):
        assert np.array_equal(_read(d, name, dt), want[key]), name
    s = json.load(open(os.path.join(d, "summary.json")))
    assert s["iterations"] == golden_index()["small"]["iterations"]
