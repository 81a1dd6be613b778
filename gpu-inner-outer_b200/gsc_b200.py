"""Python binding of the B200 grid symbolic-control library (include/gsc_b200.h).

The functions here mirror the reference's entry points
(include/gsc/cuda_api.hpp:87-88: ``cuda_backend_compiled`` and
``run_case_cuda_u32``) over the C ABI of ``libgsc_b200.so``.  There is no
CPU fallback: if the library is missing, or no CUDA device is present, the
calls raise.
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgsc_b200.so")

METHOD_AUTO, METHOD_STORED, METHOD_FUSED = 0, 1, 2
SOLVE_GRAPH = 1
SOLVE_PROFILE = 2
CONSTRAINTS = {"none": 0, "hyperbolic": 1, "elliptic": 2, "quadric": 3}
MESSAGES = {
    0: "",
    1: "all candidate states obtained a controller",
    2: "iteration stalled before candidate closure",
    3: "maximum iterations reached",
}
STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "unsupported",
    5: "no CUDA device found", 6: "candidate set contains invalid states", 7: "device wait timed out",
}
INVALID32 = 0xFFFFFFFF


class GscError(RuntimeError):
    def __init__(self, status, detail=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}" + (f": {detail}" if detail else ""))


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("state_lb", ctypes.c_double * 4), ("state_ub", ctypes.c_double * 4), ("state_eta", ctypes.c_double * 4),
        ("wrap_dim", ctypes.c_int32),
        ("input_lb", ctypes.c_double * 2), ("input_ub", ctypes.c_double * 2), ("input_eta", ctypes.c_double * 2),
        ("sample_time", ctypes.c_double), ("integration_substeps", ctypes.c_uint32),
    ]


class QueryDesc(ctypes.Structure):
    _fields_ = [
        ("disturbance_half_width", ctypes.c_double * 4),
        ("constraint_kind", ctypes.c_int32), ("constraint_params", ctypes.c_double * 4),
        ("map_lb", ctypes.c_double * 4), ("map_ub", ctypes.c_double * 4),
        ("obstacle_count", ctypes.c_uint32), ("obstacles", ctypes.c_void_p),
        ("candidate_kind", ctypes.c_int32), ("candidate", ctypes.c_double * 8),
        ("max_iterations", ctypes.c_uint32),
        ("safe_mask", ctypes.c_void_p), ("safe_mask_rank", ctypes.c_int32),
        ("valid_mask", ctypes.c_void_p), ("candidate_mask", ctypes.c_void_p),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("valid_mask", ctypes.c_void_p), ("candidate_mask", ctypes.c_void_p), ("reachable_mask", ctypes.c_void_p),
        ("controller", ctypes.c_void_p), ("reach_step", ctypes.c_void_p),
        ("iter_new_reachable", ctypes.c_void_p), ("iter_new_certified", ctypes.c_void_p),
        ("iter_capacity", ctypes.c_uint32),
        ("shape", ctypes.c_uint32 * 4), ("input_shape", ctypes.c_uint32 * 2),
        ("states", ctypes.c_uint64), ("inputs", ctypes.c_uint64), ("pairs", ctypes.c_uint64),
        ("iterations", ctypes.c_uint32), ("converged", ctypes.c_int32), ("message", ctypes.c_int32),
        ("reachable_states", ctypes.c_uint64), ("certified_candidates", ctypes.c_uint64),
        ("candidate_count", ctypes.c_uint64), ("valid_count", ctypes.c_uint64),
    ]


class Timings(ctypes.Structure):
    _fields_ = [
        ("abstraction_ms", ctypes.c_double), ("prepare_ms", ctypes.c_double), ("solve_ms", ctypes.c_double),
        ("readback_ms", ctypes.c_double), ("device_bytes", ctypes.c_uint64), ("method", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32), ("iterations", ctypes.c_uint32), ("sat_launches", ctypes.c_uint32),
        ("sat_kernel_ms", ctypes.c_double), ("scan_kernel_ms", ctypes.c_double), ("pair_tests", ctypes.c_uint64),
        ("aux_count", ctypes.c_uint64), ("sat_threads", ctypes.c_uint32), ("max_reps", ctypes.c_uint32),
    ]


class PhaseTimings(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("abstraction_kernel_ms", "abstraction_memcpy_h2d_ms",
                                               "scatter_mask_ms")] + [
        ("scan_axis_ms", ctypes.c_double * 4)] + [
        (k, ctypes.c_double) for k in ("prefix_build_total_ms", "pair_satisfaction_ms", "reduce_inputs_ms",
                                       "iteration_memcpy_ms", "result_memcpy_d2h_ms", "total_kernel_ms",
                                       "total_memcpy_ms", "total_compute_ms")] + [
        (k, ctypes.c_uint64) for k in ("total_allocated_bytes", "peak_usage_bytes", "abstraction_bytes",
                                       "prefix_bytes", "iteration_bytes", "result_bytes")] + [
        ("profiled_iterations", ctypes.c_uint32)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("autotune", ctypes.c_uint32), ("sat_threads", ctypes.c_uint32),
                ("sat_blocks_per_sm", ctypes.c_uint32), ("chunk_words", ctypes.c_uint32),
                ("sat_warp_tasks", ctypes.c_uint32)]


class BatchReport(ctypes.Structure):
    _fields_ = [
        ("create_ms", ctypes.c_double), ("tune_ms", ctypes.c_double), ("solve_ms", ctypes.c_double),
        ("device_bytes", ctypes.c_uint64), ("instances", ctypes.c_uint32), ("max_iterations_run", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32), ("sat_threads", ctypes.c_uint32),
        ("sat_blocks_per_sm", ctypes.c_uint32), ("chunk_words", ctypes.c_uint32), ("tuned", ctypes.c_uint32),
        ("sat_warp_tasks", ctypes.c_uint32), ("pair_tests", ctypes.c_uint64),
    ]


class ServerOptions(ctypes.Structure):
    _fields_ = [("memory_budget", ctypes.c_uint64), ("max_slots", ctypes.c_uint32),
                ("iterations_per_step", ctypes.c_uint32), ("sat_threads", ctypes.c_uint32),
                ("sat_blocks_per_sm", ctypes.c_uint32), ("chunk_words", ctypes.c_uint32),
                ("sat_warp_tasks", ctypes.c_uint32)]


class ServerReport(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in (
        "submitted", "completed", "failed", "queued", "in_flight", "steps", "max_running",
        "device_bytes_budget", "device_bytes_in_use", "peak_device_bytes")]


# Every symbol include/gsc_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
SIGNATURES = {
    "gsc_cuda_backend_compiled": (ctypes.c_int, []),
    "gsc_abi_version": (ctypes.c_int, []),
    "gsc_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "gsc_message_string": (ctypes.c_char_p, [ctypes.c_int]),
    "gsc_grid_shape": (ctypes.c_int, [ctypes.POINTER(ModelDesc), _P, _P]),
    "gsc_context_create": (ctypes.c_int, [ctypes.c_int, _P, ctypes.POINTER(_P)]),
    "gsc_context_destroy": (None, [_P]),
    "gsc_last_error": (ctypes.c_char_p, [_P]),
    "gsc_context_set_memory_budget": (ctypes.c_int, [_P, ctypes.c_uint64]),
    "gsc_context_memory_in_use": (ctypes.c_uint64, [_P]),
    "gsc_context_trim": (ctypes.c_int, [_P]),
    "gsc_abstraction_create": (ctypes.c_int, [_P, ctypes.POINTER(ModelDesc), ctypes.POINTER(_P)]),
    "gsc_abstraction_destroy": (None, [_P]),
    "gsc_problem_create": (ctypes.c_int, [_P, _P, ctypes.POINTER(QueryDesc), ctypes.c_uint32, ctypes.POINTER(_P)]),
    "gsc_problem_destroy": (None, [_P]),
    "gsc_problem_solve": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "gsc_problem_read": (ctypes.c_int, [_P, ctypes.POINTER(Result)]),
    "gsc_problem_export_abstraction": (ctypes.c_int, [_P, _P, _P, _P]),
    "gsc_problem_timings": (ctypes.c_int, [_P, ctypes.POINTER(Timings)]),
    "gsc_problem_phase_timings": (ctypes.c_int, [_P, ctypes.POINTER(PhaseTimings)]),
    "gsc_problem_shard_begin": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32]),
    "gsc_problem_shard_step": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "gsc_problem_shard_words": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_uint64)]),
    "gsc_problem_shard_control": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.POINTER(ctypes.c_int)]),
    "gsc_problem_iteration_timings": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, _P, _P]),
    "gsc_run_case": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ModelDesc), ctypes.POINTER(QueryDesc),
                                    ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(Result),
                                    ctypes.POINTER(Timings)]),
    "gsc_problem_simulate": (ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_uint32, ctypes.c_uint64, _P, _P, _P]),
    "gsc_batch_create": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(ModelDesc), ctypes.POINTER(QueryDesc),
                                        ctypes.POINTER(BatchOptions), ctypes.POINTER(_P)]),
    "gsc_batch_solve": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "gsc_batch_read": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(Result)]),
    "gsc_batch_read_all": (ctypes.c_int, [_P, ctypes.POINTER(Result)]),
    "gsc_batch_run": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(ModelDesc), ctypes.POINTER(QueryDesc),
                                     ctypes.POINTER(BatchOptions), ctypes.c_uint32, ctypes.POINTER(Result)]),
    "gsc_batch_timings": (ctypes.c_int, [_P, ctypes.POINTER(BatchReport)]),
    "gsc_batch_destroy": (None, [_P]),
    "gsc_server_create": (ctypes.c_int, [_P, ctypes.POINTER(ServerOptions), ctypes.POINTER(_P)]),
    "gsc_server_submit": (ctypes.c_int, [_P, _P, ctypes.POINTER(QueryDesc), ctypes.POINTER(Result),
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "gsc_server_wait": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_double)]),
    "gsc_server_stats": (ctypes.c_int, [_P, ctypes.POINTER(ServerReport)]),
    "gsc_server_destroy": (None, [_P]),
    "gsc_fixpoint_noalloc": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_int32,
                                            _P, _P, _P, _P, _P, ctypes.c_uint32, _P, _P, _P,
                                            ctypes.POINTER(Result), _P]),
}

_lib = None


def lib():
    """Load libgsc_b200.so; raises when it was not built (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def cuda_backend_compiled() -> bool:
    return bool(lib().gsc_cuda_backend_compiled())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def model_desc(case) -> ModelDesc:
    m = ModelDesc()
    m.state_lb[:] = [float(v) for v in case["state_lb"]]
    m.state_ub[:] = [float(v) for v in case["state_ub"]]
    m.state_eta[:] = [float(v) for v in case["state_eta"]]
    m.wrap_dim = int(case.get("wrap_dim", 2))
    m.input_lb[:] = [float(v) for v in case["input_lb"]]
    m.input_ub[:] = [float(v) for v in case["input_ub"]]
    m.input_eta[:] = [float(v) for v in case["input_eta"]]
    m.sample_time = float(case["sample_time"])
    m.integration_substeps = int(case["integration_substeps"])
    return m


class _Query:
    """A QueryDesc plus the host arrays it points to (kept alive with it)."""

    def __init__(self, case, safe_mask=None, safe_rank=0, valid_mask=None, candidate_mask=None):
        q = QueryDesc()
        q.disturbance_half_width[:] = [float(v) for v in case["disturbance_half_width"]]
        q.constraint_kind = CONSTRAINTS[case.get("constraint", "none")]
        cp = list(case.get("constraint_params", [0.0] * 4)) + [0.0] * 4
        q.constraint_params[:] = [float(v) for v in cp[:4]]
        q.map_lb[:] = [float(v) for v in case.get("map_lb", case["state_lb"])]
        q.map_ub[:] = [float(v) for v in case.get("map_ub", case["state_ub"])]
        obs = case.get("obstacles", [])
        self.obstacles = np.ascontiguousarray(np.array(obs, dtype=np.float64).reshape(-1, 8)) if obs else None
        q.obstacle_count = len(obs)
        q.obstacles = _ptr(self.obstacles)
        if case.get("candidate", "rect") == "rect":
            q.candidate_kind = 0
            q.candidate[:] = [float(v) for v in list(case["candidate_lb"]) + list(case["candidate_ub"])]
        else:
            q.candidate_kind = 1
            e = list(case["candidate_ellipse"]) + [0.0] * 8
            q.candidate[:] = [float(v) for v in e[:8]]
        q.max_iterations = int(case["max_iterations"])
        self.safe = np.ascontiguousarray(safe_mask, dtype=np.uint8) if safe_mask is not None else None
        self.valid = np.ascontiguousarray(valid_mask, dtype=np.uint8) if valid_mask is not None else None
        self.cand = np.ascontiguousarray(candidate_mask, dtype=np.uint8) if candidate_mask is not None else None
        q.safe_mask = _ptr(self.safe)
        q.safe_mask_rank = int(safe_rank) if self.safe is not None else 0
        q.valid_mask = _ptr(self.valid)
        q.candidate_mask = _ptr(self.cand)
        self.desc = q


def grid_shape(case):
    s = (ctypes.c_uint32 * 4)()
    u = (ctypes.c_uint32 * 2)()
    m = model_desc(case)
    st = lib().gsc_grid_shape(ctypes.byref(m), s, u)
    if st != 0:
        raise GscError(st)
    return tuple(s), tuple(u)


class Context:
    """A device + stream.  Abstractions and problems made from it are closed
    (problems first) when the context closes, since the library requires a
    context to outlive everything created from it."""

    def __init__(self, device=0, stream=None):
        self._children = weakref.WeakSet()
        self.device = int(device)
        self._h = ctypes.c_void_p()
        st = lib().gsc_context_create(int(device), ctypes.c_void_p(stream) if stream else None, ctypes.byref(self._h))
        if st != 0:
            raise GscError(st)

    def error(self):
        return lib().gsc_last_error(self._h).decode()

    def check(self, st):
        if st != 0:
            raise GscError(st, self.error())

    def set_memory_budget(self, nbytes):
        self.check(lib().gsc_context_set_memory_budget(self._h, int(nbytes)))

    def memory_in_use(self):
        return int(lib().gsc_context_memory_in_use(self._h))

    def trim(self):
        """Return the pool regions no handle uses to the driver."""
        self.check(lib().gsc_context_trim(self._h))

    def close(self):
        if self._h:
            kids = list(self._children)
            for k in kids:
                if isinstance(k, (Problem, Server, Batch)):
                    k.close()
            for k in kids:
                k.close()
            lib().gsc_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Abstraction:
    def __init__(self, ctx: Context, case):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        self.model = model_desc(case)
        ctx.check(lib().gsc_abstraction_create(ctx._h, ctypes.byref(self.model), ctypes.byref(self._h)))
        ctx._children.add(self)

    def close(self):
        if self._h:
            lib().gsc_abstraction_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Problem:
    def __init__(self, ctx: Context, abs_: Abstraction, case, method=METHOD_AUTO, **masks):
        self.ctx = ctx
        self.abs = abs_
        self._h = ctypes.c_void_p()
        self.query = _Query(case, **masks)
        self.states = int(np.prod(grid_shape(case)[0], dtype=np.uint64))
        ctx.check(lib().gsc_problem_create(ctx._h, abs_._h, ctypes.byref(self.query.desc), int(method),
                                           ctypes.byref(self._h)))
        ctx._children.add(self)

    def solve(self, graph=False, profile=False):
        flags = (SOLVE_GRAPH if graph else 0) | (SOLVE_PROFILE if profile else 0)
        self.ctx.check(lib().gsc_problem_solve(self._h, flags))

    def timings(self) -> dict:
        t = Timings()
        self.ctx.check(lib().gsc_problem_timings(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in Timings._fields_}

    def read(self, iter_capacity=4096, masks=True, out=None) -> dict:
        return _read_result(lambda r: lib().gsc_problem_read(self._h, r), self.ctx, iter_capacity, masks, out,
                            self.states)

    def phase_timings(self) -> dict:
        """Per-phase times and memory in the reference's report terms
        (gsc_problem_phase_timings), with the per-iteration times of the last
        profiled solve under ``iterations``."""
        t = PhaseTimings()
        self.ctx.check(lib().gsc_problem_phase_timings(self._h, ctypes.byref(t)))
        out = {k: (list(getattr(t, k)) if k == "scan_axis_ms" else getattr(t, k)) for k, _ in PhaseTimings._fields_}
        n = t.profiled_iterations
        cols = [np.zeros(n) for _ in range(4)]
        self.ctx.check(lib().gsc_problem_iteration_timings(self._h, n, *[_ptr(c) for c in cols]))
        out["iterations"] = {k: c for k, c in zip(("iteration_ms", "prefix_build_ms", "satisfaction_ms",
                                                   "reduction_ms"), cols)}
        return out

    def simulate(self, x0, steps, seed, trajectories=True) -> dict:
        """Closed-loop trajectories under the solved controller from each row
        of x0 ([n][4]): ``trajectories`` [n][steps+1][4] (when asked),
        ``final_states`` [n][4] and ``steps_done`` [n]."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, 4)
        n = x0.shape[0]
        tr = np.zeros((n, steps + 1, 4)) if trajectories else None
        fin = np.zeros((n, 4))
        done = np.zeros(n, np.uint32)
        self.ctx.check(lib().gsc_problem_simulate(self._h, n, _ptr(x0), int(steps), int(seed), _ptr(tr), _ptr(fin),
                                                  _ptr(done)))
        out = {"final_states": fin, "steps_done": done}
        if trajectories:
            out["trajectories"] = tr
        return out

    def export_abstraction(self):
        probe = Result()
        self.ctx.check(lib().gsc_problem_read(self._h, ctypes.byref(probe)))
        P = int(probe.pairs)
        mn = np.zeros(P, np.uint32)
        mx = np.zeros(P, np.uint32)
        v = np.zeros(P, np.uint8)
        self.ctx.check(lib().gsc_problem_export_abstraction(self._h, _ptr(mn), _ptr(mx), _ptr(v)))
        return mn, mx, v

    def close(self):
        if self._h:
            lib().gsc_problem_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _read_result(call, ctx, iter_capacity=4096, masks=True, out=None, states=None) -> dict:
    """Run a gsc_*_read call (after a shape probe when the state count is not
    given) and return the result as a dict of numpy arrays and scalars.
    ``out`` may supply the five arrays (e.g. views of pinned host memory)."""
    r = Result()
    if states is None:
        probe = Result()
        ctx.check(call(ctypes.byref(probe)))
        states = int(probe.states)
    S = int(states)
    if out is not None:
        out = dict(out)
        for k, v in out.items():
            if v.size != S or not v.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out[{k}] must be a contiguous array of {S} elements")
            setattr(r, k, _ptr(v))
    elif masks:
        out = {
            "valid_mask": np.zeros(S, np.uint8), "candidate_mask": np.zeros(S, np.uint8),
            "reachable_mask": np.zeros(S, np.uint8), "controller": np.zeros(S, np.uint32),
            "reach_step": np.zeros(S, np.uint32),
        }
        for k, v in out.items():
            setattr(r, k, _ptr(v))
    else:
        out = {}
    nr = np.zeros(iter_capacity, np.uint64)
    nc = np.zeros(iter_capacity, np.uint64)
    r.iter_new_reachable = _ptr(nr)
    r.iter_new_certified = _ptr(nc)
    r.iter_capacity = iter_capacity
    ctx.check(call(ctypes.byref(r)))
    return _result_dict(r, out, nr, nc, iter_capacity)


def _result_dict(r, out, nr, nc, iter_capacity):
    it = int(r.iterations)
    out.update({
        "shape": tuple(r.shape), "input_shape": tuple(r.input_shape), "states": int(r.states),
        "inputs": int(r.inputs), "pairs": int(r.pairs), "iterations": it, "converged": bool(r.converged),
        "message": MESSAGES[int(r.message)], "reachable_states": int(r.reachable_states),
        "certified_candidates": int(r.certified_candidates), "candidate_count": int(r.candidate_count),
        "valid_count": int(r.valid_count), "iter_new_reachable": nr[:min(it, iter_capacity)].copy(),
        "iter_new_certified": nc[:min(it, iter_capacity)].copy(),
    })
    return out


class Batch:
    """Many independent instances (each a case dict: model + query) set up
    and solved together (gsc_batch_*).  ``masks`` optionally gives, per
    instance, the keyword masks a Problem takes."""

    def __init__(self, ctx: Context, cases, autotune=False, sat_threads=0, sat_blocks_per_sm=0, chunk_words=0,
                 masks=None, sat_warp_tasks=False):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        n = len(cases)
        self.queries = [_Query(c, **((masks or [{}] * n)[i] or {})) for i, c in enumerate(cases)]
        self.models = (ModelDesc * n)(*[model_desc(c) for c in cases])
        self.qdescs = (QueryDesc * n)(*[q.desc for q in self.queries])
        opt = BatchOptions(int(bool(autotune)), int(sat_threads), int(sat_blocks_per_sm), int(chunk_words),
                           int(bool(sat_warp_tasks)))
        ctx.check(lib().gsc_batch_create(ctx._h, n, self.models, self.qdescs, ctypes.byref(opt),
                                         ctypes.byref(self._h)))
        self.count = n
        self.states = [int(np.prod(grid_shape(c)[0], dtype=np.uint64)) for c in cases]
        ctx._children.add(self)

    def solve(self, graph=True):
        self.ctx.check(lib().gsc_batch_solve(self._h, SOLVE_GRAPH if graph else 0))

    def read(self, index, iter_capacity=4096, masks=True, out=None) -> dict:
        return _read_result(lambda r: lib().gsc_batch_read(self._h, int(index), r), self.ctx, iter_capacity, masks,
                            out, self.states[int(index)])

    def read_all(self, outs=None, iter_capacity=4096) -> list:
        """Every instance with one batched read (gsc_batch_read_all); ``outs``
        may supply each instance's five arrays."""
        n = self.count
        rs = (Result * n)()
        keep = []
        for i in range(n):
            S = self.states[i]
            o = dict(outs[i]) if outs is not None else {
                "valid_mask": np.zeros(S, np.uint8), "candidate_mask": np.zeros(S, np.uint8),
                "reachable_mask": np.zeros(S, np.uint8), "controller": np.zeros(S, np.uint32),
                "reach_step": np.zeros(S, np.uint32)}
            for k, v in o.items():
                if v.size != S or not v.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"outs[{i}][{k}] must be a contiguous array of {S} elements")
                setattr(rs[i], k, _ptr(v))
            nr = np.zeros(iter_capacity, np.uint64)
            nc = np.zeros(iter_capacity, np.uint64)
            rs[i].iter_new_reachable = _ptr(nr)
            rs[i].iter_new_certified = _ptr(nc)
            rs[i].iter_capacity = iter_capacity
            keep.append((o, nr, nc))
        self.ctx.check(lib().gsc_batch_read_all(self._h, rs))
        return [_result_dict(rs[i], keep[i][0], keep[i][1], keep[i][2], iter_capacity) for i in range(n)]

    def report(self) -> dict:
        t = BatchReport()
        self.ctx.check(lib().gsc_batch_timings(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in BatchReport._fields_}

    def close(self):
        if self._h:
            lib().gsc_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_batch(ctx: Context, cases, outs=None, autotune=True, part_instances=0, iter_capacity=4096, sat_threads=0,
              sat_blocks_per_sm=0, chunk_words=0, sat_warp_tasks=False) -> list:
    """Set up, solve and read many instances in one pipelined call
    (gsc_batch_run): parts of ``part_instances`` instances overlap their
    set-up, solve and copies.  ``outs`` may supply each instance's five
    arrays (pinned memory keeps the copies asynchronous)."""
    n = len(cases)
    queries = [_Query(c) for c in cases]
    models = (ModelDesc * n)(*[model_desc(c) for c in cases])
    qdescs = (QueryDesc * n)(*[q.desc for q in queries])
    opt = BatchOptions(int(bool(autotune)), int(sat_threads), int(sat_blocks_per_sm), int(chunk_words),
                       int(bool(sat_warp_tasks)))
    rs = (Result * n)()
    keep = []
    nr_all = np.zeros((n, iter_capacity), np.uint64)
    nc_all = np.zeros((n, iter_capacity), np.uint64)
    shape, ishape = (ctypes.c_uint32 * 4)(), (ctypes.c_uint32 * 2)()
    for i, c in enumerate(cases):
        st = lib().gsc_grid_shape(ctypes.byref(models[i]), shape, ishape)
        if st != 0:
            raise GscError(st, f"instance {i}")
        S = shape[0] * shape[1] * shape[2] * shape[3]
        o = dict(outs[i]) if outs is not None else {
            "valid_mask": np.zeros(S, np.uint8), "candidate_mask": np.zeros(S, np.uint8),
            "reachable_mask": np.zeros(S, np.uint8), "controller": np.zeros(S, np.uint32),
            "reach_step": np.zeros(S, np.uint32)}
        for k, v in o.items():
            if v.size != S or not v.flags["C_CONTIGUOUS"]:
                raise ValueError(f"outs[{i}][{k}] must be a contiguous array of {S} elements")
            setattr(rs[i], k, _ptr(v))
        nr, nc = nr_all[i], nc_all[i]
        rs[i].iter_new_reachable = _ptr(nr)
        rs[i].iter_new_certified = _ptr(nc)
        rs[i].iter_capacity = iter_capacity
        keep.append((o, nr, nc))
    ctx.check(lib().gsc_batch_run(ctx._h, n, models, qdescs, ctypes.byref(opt), int(part_instances), rs))
    return [_result_dict(rs[i], keep[i][0], keep[i][1], keep[i][2], iter_capacity) for i in range(n)]


class Server:
    """The serving loop (gsc_server_*): K-invariance queries against resident
    abstractions, admitted by a device-memory budget and iterated together
    as they arrive.  ``submit`` returns a ticket; ``wait`` returns the result
    dict (as Problem.read) plus ``status`` and ``latency_ms``.  Result arrays
    may be supplied through ``out`` (e.g. views of pinned host memory, which
    lets the copies overlap the device work); they must stay alive until the
    ticket is waited for, which this object guarantees for the arrays it
    allocates itself."""

    def __init__(self, ctx: Context, memory_budget=0, max_slots=0, iterations_per_step=0, sat_threads=0,
                 sat_blocks_per_sm=0, chunk_words=0, sat_warp_tasks=False):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        opt = ServerOptions(int(memory_budget), int(max_slots), int(iterations_per_step), int(sat_threads),
                            int(sat_blocks_per_sm), int(chunk_words), int(bool(sat_warp_tasks)))
        ctx.check(lib().gsc_server_create(ctx._h, ctypes.byref(opt), ctypes.byref(self._h)))
        self._pending = {}
        ctx._children.add(self)

    def submit(self, abstraction: Abstraction, case, out=None, iter_capacity=4096, **masks) -> int:
        q = _Query(case, **masks)
        s, _ = grid_shape(case)
        S = int(np.prod(s, dtype=np.uint64))
        if out is None:
            out = {
                "valid_mask": np.zeros(S, np.uint8), "candidate_mask": np.zeros(S, np.uint8),
                "reachable_mask": np.zeros(S, np.uint8), "controller": np.zeros(S, np.uint32),
                "reach_step": np.zeros(S, np.uint32),
            }
        r = Result()
        for k, v in out.items():
            setattr(r, k, _ptr(v))
        nr = np.zeros(iter_capacity, np.uint64)
        nc = np.zeros(iter_capacity, np.uint64)
        r.iter_new_reachable = _ptr(nr)
        r.iter_new_certified = _ptr(nc)
        r.iter_capacity = iter_capacity
        t = ctypes.c_uint64()
        self.ctx.check(lib().gsc_server_submit(self._h, abstraction._h, ctypes.byref(q.desc), ctypes.byref(r),
                                               ctypes.byref(t)))
        self._pending[int(t.value)] = (q, r, out, nr, nc)
        return int(t.value)

    def wait(self, ticket, timeout_ms=-1, check=True) -> dict:
        st = ctypes.c_int()
        lat = ctypes.c_double()
        rc = lib().gsc_server_wait(self._h, int(ticket), int(timeout_ms), ctypes.byref(st), ctypes.byref(lat))
        if rc != 0:
            raise GscError(rc)
        q, r, out, nr, nc = self._pending.pop(int(ticket))
        if check and st.value != 0:
            raise GscError(st.value)
        it = int(r.iterations)
        res = dict(out)
        res.update({
            "status": int(st.value), "latency_ms": float(lat.value),
            "shape": tuple(r.shape), "input_shape": tuple(r.input_shape), "states": int(r.states),
            "inputs": int(r.inputs), "pairs": int(r.pairs), "iterations": it, "converged": bool(r.converged),
            "message": MESSAGES.get(int(r.message), ""), "reachable_states": int(r.reachable_states),
            "certified_candidates": int(r.certified_candidates), "candidate_count": int(r.candidate_count),
            "valid_count": int(r.valid_count), "iter_new_reachable": nr[:min(it, len(nr))].copy(),
            "iter_new_certified": nc[:min(it, len(nc))].copy(),
        })
        return res

    def stats(self) -> dict:
        t = ServerReport()
        self.ctx.check(lib().gsc_server_stats(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in ServerReport._fields_}

    def close(self):
        if self._h:
            lib().gsc_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_case(case, method=METHOD_AUTO, graph=False, device=0, iter_capacity=4096, out=None, **masks) -> dict:
    """One-shot run through ``gsc_run_case`` (the run_case_cuda_u32 replacement):
    host description in, host arrays out.  ``out`` may supply the five output
    arrays (e.g. views of pinned memory)."""
    L = lib()
    m = model_desc(case)
    q = _Query(case, **masks)
    s, u = grid_shape(case)
    S = int(np.prod(s, dtype=np.uint64))
    if out is None:
        out = {
            "valid_mask": np.zeros(S, np.uint8), "candidate_mask": np.zeros(S, np.uint8),
            "reachable_mask": np.zeros(S, np.uint8), "controller": np.zeros(S, np.uint32),
            "reach_step": np.zeros(S, np.uint32),
        }
    else:
        for k, dt in (("valid_mask", np.uint8), ("candidate_mask", np.uint8), ("reachable_mask", np.uint8),
                      ("controller", np.uint32), ("reach_step", np.uint32)):
            a = out[k]
            if a.dtype != dt or a.size != S or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out[{k}] must be a contiguous {np.dtype(dt).name} array of {S} elements")
        out = dict(out)
    r = Result()
    for k, v in out.items():
        setattr(r, k, _ptr(v))
    nr = np.zeros(iter_capacity, np.uint64)
    nc = np.zeros(iter_capacity, np.uint64)
    r.iter_new_reachable = _ptr(nr)
    r.iter_new_certified = _ptr(nc)
    r.iter_capacity = iter_capacity
    t = Timings()
    st = L.gsc_run_case(int(device), ctypes.byref(m), ctypes.byref(q.desc), int(method),
                        SOLVE_GRAPH if graph else 0, ctypes.byref(r), ctypes.byref(t))
    if st != 0:
        raise GscError(st)
    it = int(r.iterations)
    out.update({
        "shape": tuple(r.shape), "input_shape": tuple(r.input_shape), "states": int(r.states),
        "inputs": int(r.inputs), "pairs": int(r.pairs), "iterations": it, "converged": bool(r.converged),
        "message": MESSAGES[int(r.message)], "reachable_states": int(r.reachable_states),
        "certified_candidates": int(r.certified_candidates), "candidate_count": int(r.candidate_count),
        "valid_count": int(r.valid_count), "iter_new_reachable": nr[:min(it, iter_capacity)].copy(),
        "iter_new_certified": nc[:min(it, iter_capacity)].copy(),
        "timings": {k: getattr(t, k) for k, _ in Timings._fields_},
    })
    return out
