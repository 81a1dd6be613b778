"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle (oracle/gsc_oracle.c) restates the reference CPU method; the
reference itself, compiled from its sources, is oracle/_ref/gsc_ref.  Only the
tests, ``__graft_entry__.smoke()`` and the bench's CPU-baseline leg use this
module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "gsc_ref")

MAX_OBSTACLES = 16
MESSAGES = {
    0: "",
    1: "all candidate states obtained a controller",
    2: "iteration stalled before candidate closure",
    3: "maximum iterations reached",
}


class OrcCase(ctypes.Structure):
    _fields_ = [
        ("state_lb", ctypes.c_double * 4),
        ("state_ub", ctypes.c_double * 4),
        ("state_eta", ctypes.c_double * 4),
        ("wrap_dim", ctypes.c_int32),
        ("input_lb", ctypes.c_double * 2),
        ("input_ub", ctypes.c_double * 2),
        ("input_eta", ctypes.c_double * 2),
        ("sample_time", ctypes.c_double),
        ("substeps", ctypes.c_uint32),
        ("dhw", ctypes.c_double * 4),
        ("constraint_kind", ctypes.c_int32),
        ("cparam", ctypes.c_double * 4),
        ("map_lb", ctypes.c_double * 4),
        ("map_ub", ctypes.c_double * 4),
        ("n_obstacles", ctypes.c_int32),
        ("obstacles", (ctypes.c_double * 8) * MAX_OBSTACLES),
        ("candidate_kind", ctypes.c_int32),
        ("cand", ctypes.c_double * 8),
        ("max_iterations", ctypes.c_uint32),
    ]


class OrcSummary(ctypes.Structure):
    _fields_ = [
        ("shape", ctypes.c_uint32 * 4),
        ("input_shape", ctypes.c_uint32 * 2),
        ("states", ctypes.c_uint64),
        ("inputs", ctypes.c_uint64),
        ("pairs", ctypes.c_uint64),
        ("iterations", ctypes.c_uint32),
        ("converged", ctypes.c_int32),
        ("message", ctypes.c_int32),
        ("reachable_states", ctypes.c_uint64),
        ("certified_candidates", ctypes.c_uint64),
        ("candidate_count", ctypes.c_uint64),
        ("valid_count", ctypes.c_uint64),
        ("valid_pairs", ctypes.c_uint64),
        ("abstraction_ms", ctypes.c_double),
        ("solve_ms", ctypes.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, os.path.join(HERE, "liboracle.so")], check=True,
                           stdout=subprocess.DEVNULL)
        _lib = ctypes.CDLL(LIB_PATH)
        p = ctypes.POINTER
        _lib.orc_shapes.argtypes = [p(OrcCase), p(ctypes.c_uint32), p(ctypes.c_uint32)]
        _lib.orc_masks.argtypes = [p(OrcCase), ctypes.c_void_p, ctypes.c_void_p]
        _lib.orc_abstraction.argtypes = [p(OrcCase), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int]
        _lib.orc_prefix.argtypes = [p(ctypes.c_uint32), ctypes.c_void_p, ctypes.c_void_p]
        _lib.orc_query.restype = ctypes.c_uint64
        _lib.orc_query.argtypes = [p(ctypes.c_uint32), ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                   ctypes.c_uint32]
        _lib.orc_solve.argtypes = [p(OrcCase)] + [ctypes.c_void_p] * 7 + [ctypes.c_uint32, p(OrcSummary),
                                                                           ctypes.c_int]
        _lib.orc_spot_step.argtypes = [p(OrcCase)] + [ctypes.c_void_p] * 5 + [
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_int]
    return _lib


def to_struct(case) -> OrcCase:
    """Pack a ``gsc_b200`` case description (a dict) into the oracle struct."""
    c = OrcCase()
    for k in ("state_lb", "state_ub", "state_eta"):
        getattr(c, k)[:] = [float(v) for v in case[k]]
    c.wrap_dim = int(case.get("wrap_dim", 2))
    for k in ("input_lb", "input_ub", "input_eta"):
        getattr(c, k)[:] = [float(v) for v in case[k]]
    c.sample_time = float(case["sample_time"])
    c.substeps = int(case["integration_substeps"])
    c.dhw[:] = [float(v) for v in case["disturbance_half_width"]]
    kinds = {"none": 0, "hyperbolic": 1, "elliptic": 2, "quadric": 3}
    c.constraint_kind = kinds[case.get("constraint", "none")]
    cp = list(case.get("constraint_params", [0.0, 0.0, 0.0, 0.0])) + [0.0] * 4
    c.cparam[:] = [float(v) for v in cp[:4]]
    c.map_lb[:] = [float(v) for v in case.get("map_lb", case["state_lb"])]
    c.map_ub[:] = [float(v) for v in case.get("map_ub", case["state_ub"])]
    obs = case.get("obstacles", [])
    assert len(obs) <= MAX_OBSTACLES
    c.n_obstacles = len(obs)
    for i, o in enumerate(obs):
        c.obstacles[i][:] = [float(v) for v in o]
    if case.get("candidate", "rect") == "rect":
        c.candidate_kind = 0
        c.cand[:] = [float(v) for v in list(case["candidate_lb"]) + list(case["candidate_ub"])]
    else:
        c.candidate_kind = 1
        e = list(case["candidate_ellipse"]) + [0.0] * 8
        c.cand[:] = [float(v) for v in e[:8]]
    c.max_iterations = int(case["max_iterations"])
    return c


def shapes(case):
    s = (ctypes.c_uint32 * 4)()
    u = (ctypes.c_uint32 * 2)()
    c = to_struct(case)
    if lib().orc_shapes(ctypes.byref(c), s, u) != 0:
        raise ValueError("invalid grid")
    return tuple(s), tuple(u)


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def masks(case):
    (shape, _) = shapes(case)
    S = int(np.prod(shape, dtype=np.uint64))
    valid = np.zeros(S, np.uint8)
    cand = np.zeros(S, np.uint8)
    c = to_struct(case)
    rc = lib().orc_masks(ctypes.byref(c), _ptr(valid), _ptr(cand))
    if rc != 0:
        raise ValueError("candidate set contains invalid states" if rc == -1 else "invalid grid")
    return valid, cand


def abstraction(case, nthreads: int = 0):
    """Per-pair (min_flat, max_flat, valid), pair = state * M + input."""
    shape, ishape = shapes(case)
    P = int(np.prod(shape, dtype=np.uint64)) * ishape[0] * ishape[1]
    mn = np.zeros(P, np.uint32)
    mx = np.zeros(P, np.uint32)
    pv = np.zeros(P, np.uint8)
    c = to_struct(case)
    lib().orc_abstraction(ctypes.byref(c), _ptr(mn), _ptr(mx), _ptr(pv), nthreads)
    return mn, mx, pv


def prefix(shape, mask: np.ndarray) -> np.ndarray:
    s = (ctypes.c_uint32 * 4)(*shape)
    T = int(np.prod([n + 1 for n in shape], dtype=np.uint64))
    out = np.zeros(T, np.uint64)
    lib().orc_prefix(s, _ptr(np.ascontiguousarray(mask, dtype=np.uint8)), _ptr(out))
    return out


def solve(case, nthreads: int = 0, iter_cap: int = 4096) -> dict:
    shape, ishape = shapes(case)
    S = int(np.prod(shape, dtype=np.uint64))
    out = {
        "valid_mask": np.zeros(S, np.uint8),
        "candidate_mask": np.zeros(S, np.uint8),
        "reachable_mask": np.zeros(S, np.uint8),
        "controller": np.zeros(S, np.uint32),
        "reach_step": np.zeros(S, np.uint32),
    }
    nr = np.zeros(iter_cap, np.uint64)
    nc = np.zeros(iter_cap, np.uint64)
    sm = OrcSummary()
    c = to_struct(case)
    rc = lib().orc_solve(ctypes.byref(c), _ptr(out["valid_mask"]), _ptr(out["candidate_mask"]),
                         _ptr(out["reachable_mask"]), _ptr(out["controller"]), _ptr(out["reach_step"]),
                         _ptr(nr), _ptr(nc), iter_cap, ctypes.byref(sm), nthreads)
    if rc != 0:
        raise ValueError(f"oracle solve failed: {rc}")
    it = sm.iterations
    out.update({
        "shape": tuple(sm.shape), "input_shape": tuple(sm.input_shape), "states": sm.states,
        "inputs": sm.inputs, "pairs": sm.pairs, "iterations": it, "converged": bool(sm.converged),
        "message": MESSAGES[sm.message], "reachable_states": sm.reachable_states,
        "certified_candidates": sm.certified_candidates, "candidate_count": sm.candidate_count,
        "valid_count": sm.valid_count, "valid_pairs": sm.valid_pairs,
        "iter_new_reachable": nr[:it].copy(), "iter_new_certified": nc[:it].copy(),
        "abstraction_ms": sm.abstraction_ms, "solve_ms": sm.solve_ms,
    })
    return out


def spot_step(case, valid, cand, reach_prev, ctl_prev, step_prev, it, states, nthreads: int = 0):
    """One Jacobi iteration recomputed for the listed states only."""
    states = np.ascontiguousarray(states, dtype=np.uint64)
    n = states.size
    rn = np.zeros(n, np.uint8)
    ct = np.zeros(n, np.uint32)
    st = np.zeros(n, np.uint32)
    c = to_struct(case)
    arrs = [np.ascontiguousarray(a) for a in (valid, cand, reach_prev, ctl_prev, step_prev)]
    rc = lib().orc_spot_step(ctypes.byref(c), *[_ptr(a) for a in arrs], it, _ptr(states), n, _ptr(rn),
                             _ptr(ct), _ptr(st), nthreads)
    if rc != 0:
        raise ValueError(f"spot step failed: {rc}")
    return rn, ct, st


def run_reference(case, outdir: str | None = None) -> dict:
    """Run the reference's own CPU method (oracle/_ref/gsc_ref full)."""
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    shape, ishape = shapes(case)
    S = int(np.prod(shape, dtype=np.uint64))
    tmp = tempfile.TemporaryDirectory() if outdir is None else None
    d = tmp.name if tmp else outdir
    try:
        cpath = os.path.join(d, "case.bin")
        with open(cpath, "wb") as f:
            f.write(bytes(to_struct(case)))
        proc = subprocess.run([REF_BIN, "full", cpath, d], check=True, capture_output=True, text=True)
        out = {
            "valid_mask": np.fromfile(os.path.join(d, "valid.u8"), np.uint8),
            "candidate_mask": np.fromfile(os.path.join(d, "candidate.u8"), np.uint8),
            "reachable_mask": np.fromfile(os.path.join(d, "reachable.u8"), np.uint8),
            "controller": np.fromfile(os.path.join(d, "controller.u32"), np.uint32),
            "reach_step": np.fromfile(os.path.join(d, "reach_step.u32"), np.uint32),
        }
        if os.path.exists(os.path.join(d, "min_flat.u32")):
            out["min_flat"] = np.fromfile(os.path.join(d, "min_flat.u32"), np.uint32)
            out["max_flat"] = np.fromfile(os.path.join(d, "max_flat.u32"), np.uint32)
            out["pair_valid"] = np.fromfile(os.path.join(d, "pair_valid.u8"), np.uint8)
        assert out["valid_mask"].size == S
        nr, cov = [], []
        for line in proc.stdout.splitlines():
            m = re.match(r"iter (\d+): new_reachable=(\d+) .*\((\d+)/(\d+)\)", line)
            if m:
                nr.append(int(m.group(2)))
                cov.append(int(m.group(3)))
            if line.startswith("SUMMARY"):
                kv = dict(t.split("=") for t in line.split()[1:])
                out["iterations"] = int(kv["iterations"])
                out["converged"] = kv["converged"] == "1"
                out["reachable_states"] = int(kv["reachable"])
                out["certified_candidates"] = int(kv["certified"])
                out["valid_pairs"] = int(kv["valid_pairs"])
                out["abstraction_ms"] = float(kv["abstraction_ms"])
                out["solve_ms"] = float(kv["solve_ms"])
            if line.startswith("MESSAGE "):
                out["message"] = line[len("MESSAGE "):]
        out["iter_new_reachable"] = np.array(nr, np.uint64)
        out["iter_new_certified"] = np.diff(np.array([0] + cov, np.int64)).astype(np.uint64)
        return out
    finally:
        if tmp:
            tmp.cleanup()
