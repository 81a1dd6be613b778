#!/usr/bin/env python
"""Benchmark of the grid symbolic-control fixpoint on B200.

Metric: nominal pair-checks per second = states x inputs x iterations / fixpoint
time (the reference tests every pair every iteration, cuda/kernels.cu:668), on
the 65x65x38x25-state x 10x10-input unicycle workload (seeded synthetic grid,
no dataset).  One step = one full backward-reachability fixpoint from the
candidate set, with the abstraction and masks resident in HBM.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) every rank solves its own replica of the workload
(independent K-invariance queries shard without any exchange), the step time is
the max over ranks, and value = the pair-checks of all ranks / that time.

`--impl reference` times the reference's own CPU method (oracle/_ref/gsc_ref,
compiled from its sources) on the host cores: every step is one full-grid
fixpoint iteration of the same workload, states split over the host threads.
The default run also times the reference's own CUDA backend (oracle/_ref/
gsc_ref_gpu, built for sm_100a) on the published demo next to this library's
solve of the same case (`reference_gpu`).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu-inner-outer_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

import gsc_cases as C  # noqa: E402

REF_BIN = os.path.join(ORACLE, "_ref", "gsc_ref")
REF_GPU_BIN = os.path.join(ORACLE, "_ref", "gsc_ref_gpu")
PUBLISHED_DEMO_SOLVE_MS = 214.936   # README.md:69, RTX 4090, 12 iterations
PUBLISHED_DEMO_PAIRS = 401310000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(C.PRESETS) + ["batched", "served", "simulate"], default="demo_scale")
    ap.add_argument("--method", choices=["auto", "stored", "fused"], default="auto")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="one problem over all ranks by slice ranges (strong scaling) instead of replicas")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's CUDA backend on the published demo beside this library's")
    ap.add_argument("--e2e-steps", type=int, default=5)
    # batched / served workloads
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--queries", type=int, default=10000)
    ap.add_argument("--rates", type=str, default="0.5,0.75,0.9",
                    help="Poisson arrival rates as fractions of the measured saturation throughput")
    ap.add_argument("--serve-budget-gb", type=float, default=24.0)
    ap.add_argument("--sat-warp-tasks", type=int, default=0, choices=[0, 1],
                    help="served: one satisfaction task per warp in the serving loop's batched steps")
    ap.add_argument("--serve-iterations-per-step", type=int, default=0,
                    help="served: fixpoint iterations between the serving loop's host checks (0: the library's)")
    ap.add_argument("--serve-sat-threads", type=int, default=0, choices=[0, 64, 128, 256],
                    help="served: satisfaction block size of the serving loop's batched steps (0: the library's)")
    ap.add_argument("--serve-sat-blocks-per-sm", type=int, default=0,
                    help="served: persistent satisfaction blocks per SM (0: the library's)")
    ap.add_argument("--host-loop", action="store_true",
                    help="batched: iterate from the host instead of one CUDA graph (for per-kernel profiling)")
    ap.add_argument("--trajectories", type=int, default=1 << 20)
    ap.add_argument("--sim-steps", type=int, default=40)
    ap.add_argument("--plain-queries", type=int, default=0,
                    help="queries timed through the plain API for the sequential baseline (0 = all)")
    return ap.parse_args()


# ---- CPU and GPU: the reference's own code --------------------------------------------------

def reference_gpu_runs(case, runs):
    """The reference's own CUDA backend (cuda/kernels.cu, rebuilt for sm_100a
    by oracle/Makefile) on this GPU: one record per run_case_cuda_u32 call."""
    sys.path.insert(0, ORACLE)
    import oracle as O

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "case.bin")
        with open(path, "wb") as f:
            f.write(bytes(O.to_struct(case)))
        r = subprocess.run([REF_GPU_BIN, path, str(runs)], capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"unavailable": (r.stderr.strip().splitlines() or ["exit %d" % r.returncode])[-1]}
    recs = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    med = lambda k: statistics.median(x[k] for x in recs)
    return {"runs": len(recs), "solve_ms": med("solve_ms"), "abstraction_ms": med("abstraction_ms"),
            "total_ms": med("total_ms"), "pair_satisfaction_ms": med("pair_satisfaction_ms"),
            "prefix_build_ms": med("prefix_build_ms"), "iterations": recs[0]["iterations"],
            "reachable_states": recs[0]["reachable_states"],
            "certified_candidates": recs[0]["certified_candidates"], "message": recs[0]["message"],
            "device_bytes": recs[0]["device_bytes"],
            "note": "the reference's cuda/kernels.cu built for sm_100a, run_case_cuda_u32 on the same GPU "
                    "(solve_ms: its fixpoint loop; total_ms: with the abstraction and its copy to the host)"}


def reference_full_runs(cases, budget_ms=20000.0):
    """The reference's own CPU method as shipped (prepare_case_cpu +
    solve_backward_cpu, single-threaded: oracle/_ref/gsc_ref full) on the
    cases in order, until its own timers have counted budget_ms.  Returns the
    number of cases run and their summed abstraction + solve milliseconds."""
    sys.path.insert(0, ORACLE)
    import oracle as O

    n, total = 0, 0.0
    for c in cases:
        r = O.run_reference(c)
        total += r["abstraction_ms"] + r["solve_ms"]
        n += 1
        if total >= budget_ms:
            break
    return n, total


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_bench(case, threads, warmup, steps, single):
    """One run of `gsc_ref bench`: the reference's CPU method on the whole
    grid.  Set-up (untimed) builds the full abstraction with the reference's
    per-pair steps, its states split over `threads`; then warmup + steps
    full-grid fixpoint iterations from the start state are timed one by one
    (the reachable prefix build plus every state's body,
    reachability.hpp:53-109, states split over `threads`).  With `single` it
    also times one iteration of solve_backward_cpu itself, single-threaded as
    shipped.  Returns the parsed SETUP, STEP and SINGLE records."""
    sys.path.insert(0, ORACLE)
    import oracle as O

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "case.bin")
        with open(path, "wb") as f:
            f.write(bytes(O.to_struct(case)))
        out = subprocess.run([REF_BIN, "bench", path, str(threads), str(warmup), str(steps), "1" if single else "0"],
                             check=True, capture_output=True, text=True).stdout
    recs = {"steps": []}
    for ln in out.splitlines():
        tag, *rest = ln.split()
        kv = dict(t.split("=") for t in rest)
        if tag == "SETUP":
            recs["setup"] = kv
        elif tag == "STEP" and kv["warm"] == "0":
            recs["steps"].append({k: float(v) for k, v in kv.items()})
        elif tag == "SINGLE":
            recs["single"] = kv
    return recs


def run_reference_arm(args, case):
    """The reference's own CPU method on the host cores, on the same workload:
    every step is one full-grid fixpoint iteration (all states x all inputs),
    timed as it runs, so ms_per_step is the time each step really took and
    value = states x inputs / that time (the nominal accounting of the GPU
    arm).  A single-threaded iteration of the reference's solver as shipped
    is reported beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    metric = "fixpoint pair-checks/s"
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/gsc_ref was not built"}))
        return
    threads = cpu_threads()
    r = reference_bench(case, threads, args.warmup, args.steps, single=True)
    S, M = int(r["setup"]["states"]), int(r["setup"]["inputs"])
    step_ms = [x["step_ms"] for x in r["steps"]]
    ms = statistics.mean(step_ms)
    v = S * M / (ms * 1e-3)
    single_ms = float(r["single"]["solve_ms"])
    sample = (f"every step = one full fixpoint iteration of the {case['name']} grid ({S} states x {M} inputs) "
              f"from the start state: build_prefix_sum_cpu plus every state's body (reachability.hpp:53-109), "
              f"states split over {threads} threads; the abstraction is built once before the steps (untimed)")
    line = {
        "impl": "reference", "metric": metric, "value": v, "unit": "pair-checks/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": case["name"], "states": S, "inputs": M, "pairs": S * M,
                   "step": "one full-grid fixpoint iteration", "threads": threads,
                   "abstraction_setup_ms": float(r["setup"]["abstraction_ms"]),
                   "step_ms": {"median": statistics.median(step_ms), "min": min(step_ms), "max": max(step_ms)}},
        "cpu_baseline": {"value": v, "unit": "pair-checks/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "single_thread_as_shipped": {
            "value": S * M / (single_ms * 1e-3), "unit": "pair-checks/s", "cores": 1, "iteration_ms": single_ms,
            "note": "one iteration of the reference's solve_backward_cpu (reachability.hpp:30-155) on the same "
                    "prepared case, single-threaded as shipped"},
        "e2e": {"value": v, "unit": "pair-checks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    # The reference's CUDA backend expresses the published demo (built-in
    # hyperbolic constraint, rectangular candidate set) but not the quadric
    # safe set of the other workloads.
    if args.workload == "hyperbolic_demo" and os.path.exists(REF_GPU_BIN):
        line["reference_gpu"] = reference_gpu_runs(case, 3)
    print(json.dumps(line))


def reference_gpu_beside_ours(G, torch, dev, stream, runs=3, steps=10):
    """The published demo (examples/hyperbolic_case.cfg, 70x70x63x13 x 100)
    through the reference's own CUDA backend on this GPU, next to this
    library's fixpoint (graph solve, device events, L2 flushed) and its
    end-to-end gsc_run_case on the same case."""
    if not os.path.exists(REF_GPU_BIN):
        return {"unavailable": "oracle/_ref/gsc_ref_gpu was not built"}
    case = C.checked(C.hyperbolic_demo_case())
    ref = reference_gpu_runs(case, runs)
    if "unavailable" in ref:
        return ref
    ctx = G.Context(dev.index, stream.cuda_stream)
    absn = G.Abstraction(ctx, case)
    prob = G.Problem(ctx, absn, case, G.METHOD_AUTO)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(3):
        prob.solve(graph=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        flush.fill_(3)
        a.record(stream)
        prob.solve(graph=True)
        b.record(stream)
    torch.cuda.synchronize(dev)
    ours_ms = statistics.median(a.elapsed_time(b) for a, b in evs)
    got = prob.read(masks=False)
    prob.close()
    absn.close()
    ctx.close()
    outs = pinned_outputs(torch, int(got["states"]))
    e2e = []
    for k in range(runs + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        G.run_case(case, graph=False, device=dev.index, out=outs)
        if k:
            e2e.append((time.perf_counter() - t0) * 1e3)
    ours_e2e = statistics.median(e2e)
    same = (got["iterations"] == ref["iterations"] and got["reachable_states"] == ref["reachable_states"] and
            got["certified_candidates"] == ref["certified_candidates"])
    return {"workload": case["name"], "reference": ref,
            "ours": {"fixpoint_ms": ours_ms, "e2e_ms": ours_e2e, "iterations": got["iterations"],
                     "reachable_states": got["reachable_states"],
                     "certified_candidates": got["certified_candidates"]},
            "same_counts": same,
            "fixpoint_speedup": ref["solve_ms"] / ours_ms, "e2e_speedup": ref["total_ms"] / ours_e2e,
            "published_rtx4090_fixpoint_ms": PUBLISHED_DEMO_SOLVE_MS,
            "note": "reference: cuda/kernels.cu built for sm_100a, run_case_cuda_u32 (solve_ms = its fixpoint "
                    "loop, total_ms = the whole call with its abstraction and result copies); ours: the graph "
                    "solve with device events, and gsc_run_case end to end with the host-loop solve (host description "
                    "in, results in pinned host arrays)"}


# ---- GPU --------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.lines = []
        self.proc = None

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.15)
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_figure(tag, field, kernel, workload):
    """A per-launch figure of `kernel` on `workload` from a committed ncu
    summary (profiles/*.md lines '<tag> kernel=<k> workload=<w> <field>=<n>')."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".txt", ".md")):
            continue
        with open(os.path.join(pdir, fn)) as f:
            for ln in f:
                if ln.startswith(tag + " ") and f"kernel={kernel} " in ln and f"workload={workload} " in ln:
                    for tok in ln.split():
                        if tok.startswith(field + "="):
                            return float(tok.split("=")[1])
    return None


def ncu_traffic(kernel, workload):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)."""
    return ncu_figure("traffic", "bytes_per_launch", kernel, workload)


def issue_roofline(kernel, workload, per_launch_ms, sm_mhz, sms):
    """The kernel against its issue rate: warp instructions per launch
    (smsp__inst_executed.sum averaged over one fixpoint's launches, from a
    committed ncu summary) over the live launch time, against 4 schedulers
    per SM issuing one warp instruction per cycle at the sampled SM clock."""
    inst = ncu_figure("instructions", "warp_instructions_per_launch", kernel, workload)
    if not inst or not sm_mhz or not per_launch_ms:
        return None
    achieved = inst / (per_launch_ms * 1e-3) / 1e12
    peak = 4 * sms * sm_mhz * 1e6 / 1e12
    return {"achieved": achieved, "peak": peak, "unit": "T warp instructions/s", "frac": achieved / peak,
            "warp_instructions_per_launch": inst}


def algorithmic_bytes(method, g, timings):
    """Bytes one satisfaction launch must move, from the counters of a profiled
    solve.  stored: 8 B per streamed (state, input) box + valid, candidate,
    reachable (1 B each) and controller (4 B) per state.  fused: the x and y
    box-table rows of every processed (slice, input) plane task (4 B per entry)
    + four passes over the 32-bit bit-sliced sets (active, hit, previous and
    next reachable) per launch."""
    n0, n1, n2, n3 = g["shape"]
    S = n0 * n1 * n2 * n3
    L = max(timings["sat_launches"], 1)
    if method == 1:
        return (8.0 * timings["pair_tests"] + 7.0 * S * L) / L
    W = (n0 + 31) // 32
    words = n1 * n2 * n3 * W
    return (4.0 * (n0 + n1) * timings["aux_count"] + 16.0 * words * L) / L


def gpu_uuid(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:   # noqa: BLE001
        return None


def max_over_ranks(dist, values, device):
    """Every rank's values replaced by their maximum over the ranks (one
    all-reduce); unchanged without a process group."""
    if not dist:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_value(world, units_per_rank, ms):
    """Whole-job throughput of `world` replicas that each process
    `units_per_rank` units in `ms` milliseconds (the slowest rank's time)."""
    return world * units_per_rank / (ms * 1e-3)


def pinned_outputs(torch, S):
    """The five result arrays of one problem as numpy views of pinned memory."""
    import numpy as np

    bufs = {k: torch.empty(S * sz, dtype=torch.uint8, pin_memory=True)
            for k, sz in (("valid_mask", 1), ("candidate_mask", 1), ("reachable_mask", 1), ("controller", 4),
                          ("reach_step", 4))}
    return {k: (v.numpy() if k.endswith("mask") else v.numpy().view(np.uint32)) for k, v in bufs.items()}


def percentile(xs, q):
    import numpy as np

    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def plain_solve(G, ctx, absn, case, out):
    """One query through the plain API: problem set-up, graph solve, read."""
    p = G.Problem(ctx, absn, case, G.METHOD_FUSED)
    p.solve(graph=True)
    r = p.read(out=out)
    p.close()
    return r


def bench_batched(args):
    """64 seeded instances of uneven grid and input size (random_instance):
    value = instances/s of the batched fixpoint with everything resident
    (one step = one gsc_batch_solve of all instances, L2 flushed before each);
    e2e = instances/s of gsc_batch_create + solve + reads into pinned host
    memory; beside it the same instances one by one through the plain API
    (abstraction, problem, graph solve, read)."""
    import numpy as np
    import torch
    import gsc_b200 as G

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    cases = [C.random_instance(args.seed, i) for i in range(args.instances)]
    sizes = [int(np.prod(C.grid_shape(c)[0])) for c in cases]
    outs = [pinned_outputs(torch, S) for S in sizes]
    ctx = G.Context(0, stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    graph = not args.host_loop
    b = G.Batch(ctx, cases, autotune=True)     # tunes once; later batches of this class reuse the shapes
    rep0 = b.report()
    for _ in range(args.warmup):
        flush.fill_(1)
        b.solve(graph=graph)
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    with ClockSampler(gpu_uuid(torch, dev)) as clocks:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            evs[k][0].record(stream)
            b.solve(graph=graph)
            evs[k][1].record(stream)
        torch.cuda.synchronize(dev)
    rep = b.report()
    launches = rep["kernel_launches"] * args.steps
    step_ms = statistics.median(a.elapsed_time(c) for a, c in evs)
    b.close()

    # End to end: create + solve + read all, host wall clock.
    # End to end through gsc_batch_run: parts overlap set-up, solve and copies.
    e2e = []
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        G.run_batch(ctx, cases, outs, autotune=True)
        if k:
            e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = statistics.median(e2e)
    # The same through the three calls of one batch (create, solve, read).
    e2e_seq = []
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        bb = G.Batch(ctx, cases, autotune=True)
        bb.solve(graph=True)
        bb.read_all(outs)
        bb.close()
        if k:
            e2e_seq.append((time.perf_counter() - t0) * 1e3)
    e2e_seq_ms = statistics.median(e2e_seq)

    # Sequential plain solves of the same instances (one warm pass first).
    plain_ms, plain_dev = [], []
    for rnd in range(2):
        plain_ms, plain_dev = [], []
        for c, o in zip(cases, outs):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            a = G.Abstraction(ctx, c)
            p = G.Problem(ctx, a, c, G.METHOD_FUSED)
            p.solve(graph=True)
            p.read(out=o)
            plain_dev.append(p.timings()["solve_ms"])
            p.close()
            a.close()
            plain_ms.append((time.perf_counter() - t0) * 1e3)
    plain_total = sum(plain_ms)
    n = len(cases)
    h2d = 0
    d2h = sum(11 * S for S in sizes)
    cpu = None
    if not args.no_cpu_baseline and os.path.exists(REF_BIN):
        k, ref_ms = reference_full_runs(cases)
        cpu = {"value": k / (ref_ms * 1e-3), "unit": "instances/s", "cores": 1, "kind": "reference",
               "sample": f"the first {k} of the {n} instances, each a full run of the reference's CPU method as "
                         f"shipped (prepare_case_cpu + solve_backward_cpu, one thread): {ref_ms:.0f} ms by its own "
                         f"timers"}
    line = {
        "metric": "batched instances/s", "value": n / (step_ms * 1e-3), "unit": "instances/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 bit-sliced sets / int32 counts (f64 boxes)",
        "data": "synthetic",
        "config": {"workload": f"batched_{n}_random_instances_seed{args.seed}", "instances": n,
                   "states_total": sum(sizes), "max_iterations_run": rep["max_iterations_run"],
                   "shapes": {"sat_threads": rep["sat_threads"], "sat_blocks_per_sm": rep["sat_blocks_per_sm"],
                              "chunk_words": rep["chunk_words"], "sat_warp_tasks": rep["sat_warp_tasks"],
                              "tuned": rep0["tuned"],
                              "tune_ms": rep0["tune_ms"]},
                   "l2": "flushed before every step (256 MiB write)"},
        "e2e": {"value": n / (e2e_ms * 1e-3), "unit": "instances/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "note": "gsc_batch_run: parts of an eighth of the instances overlap set-up (abstractions + "
                        "problems), graph solve and the copies of all results into pinned memory",
                "create_solve_read_ms": e2e_seq_ms},
        "plain_sequential": {
            "e2e_instances_per_s": n / (plain_total * 1e-3), "e2e_ms_total": plain_total,
            "device_solve_ms_total": sum(plain_dev), "p50_ms": percentile(plain_ms, 50),
            "p99_ms": percentile(plain_ms, 99),
            "note": "per instance: abstraction + problem set-up + graph solve + read into pinned memory"},
        "speedup_vs_plain": {"e2e": plain_total / e2e_ms, "fixpoint": sum(plain_dev) / step_ms},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))
    ctx.close()


def bench_served(args):
    """A Poisson stream of seeded K-invariance queries (random_query: safe
    set, candidate ellipse, disturbance bound, iteration cap) against three
    resident abstractions (20x20x16x10 x 25, 65x65x38x25 x 100,
    32x32x24x16 x 64 inputs).  First all queries at once (saturation), then
    three arrival rates as fractions of that throughput; latency = scheduled
    arrival to completion.  Beside it the same queries one at a time through
    the plain API: its throughput, and its latencies measured at the same
    arrival times."""
    import queue
    import numpy as np
    import torch
    import gsc_b200 as G

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    models = {"small": C.small_case(), "demo": C.demo_scale_case(), "mid": C.serve_mid_case()}
    names = list(models)
    ctx = G.Context(0)
    absn = {k: G.Abstraction(ctx, c) for k, c in models.items()}
    S = {k: int(np.prod(C.grid_shape(c)[0])) for k, c in models.items()}
    rng = np.random.default_rng(args.seed)
    pick = rng.integers(0, 3, size=args.queries)
    qs = [(names[k], C.random_query(models[names[k]], args.seed, i)) for i, k in enumerate(pick)]
    # Pinned result buffers, recycled: at most this many queries of a model in flight.
    depth = {"small": 128, "demo": 24, "mid": 96}
    pools = {k: queue.Queue() for k in names}
    for k in names:
        for _ in range(depth[k]):
            pools[k].put(pinned_outputs(torch, S[k]))

    def run_stream(srv, arrivals):
        n = len(qs)
        submit_t = [0.0] * n
        server_lat = [0.0] * n
        tickets = [None] * n
        per_model = {k: queue.Queue() for k in names}
        errors = []

        def waiter(k):
            while True:
                item = per_model[k].get()
                if item is None:
                    return
                i, t, buf = item
                try:
                    r = srv.wait(t)
                    server_lat[i] = r["latency_ms"]
                except Exception as e:   # noqa: BLE001
                    errors.append(e)
                pools[k].put(buf)

        ths = [threading.Thread(target=waiter, args=(k,), daemon=True) for k in names]
        for th in ths:
            th.start()
        t0 = time.perf_counter()
        for i, (k, q) in enumerate(qs):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            buf = pools[k].get()
            submit_t[i] = time.perf_counter() - t0
            tickets[i] = srv.submit(absn[k], q, out=buf)
            per_model[k].put((i, tickets[i], buf))
        for k in names:
            per_model[k].put(None)
        for th in ths:
            th.join()
        total = time.perf_counter() - t0
        if errors:
            raise errors[0]
        lat = [(submit_t[i] - arrivals[i]) * 1e3 + server_lat[i] for i in range(n)]
        return total, lat

    srv = G.Server(ctx, memory_budget=int(args.serve_budget_gb * (1 << 30)), max_slots=256,
                   sat_warp_tasks=bool(args.sat_warp_tasks), iterations_per_step=args.serve_iterations_per_step,
                   sat_threads=args.serve_sat_threads, sat_blocks_per_sm=args.serve_sat_blocks_per_sm)
    # warm-up: a few queries of each model
    warm = [srv.submit(absn[k], C.random_query(models[k], args.seed + 1, i)) for i, k in enumerate(names * 4)]
    for t in warm:
        srv.wait(t)
    n = len(qs)
    with ClockSampler(gpu_uuid(torch, dev)) as clocks:
        sat_s, sat_lat = run_stream(srv, [0.0] * n)
        X = n / sat_s
        rates = []
        for f in [float(v) for v in args.rates.split(",") if v]:
            lam = f * X
            arr = np.cumsum(np.random.default_rng(args.seed + 17).exponential(1.0 / lam, size=n)).tolist()
            tot, lat = run_stream(srv, arr)
            rates.append({"fraction_of_saturation": f, "rate_qps": lam, "throughput_qps": n / tot,
                          "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "arrivals": arr})
    st = srv.stats()
    st_ips = args.serve_iterations_per_step or 2
    srv.close()

    # Sequential plain solves: service time of every query (or a prefix).
    m = args.plain_queries or n
    plain_out = {k: pinned_outputs(torch, S[k]) for k in names}
    for k in names:   # warm
        plain_solve(G, ctx, absn[k], models[k], plain_out[k])
    svc = []
    for k, q in qs[:m]:
        t0 = time.perf_counter()
        plain_solve(G, ctx, absn[k], q, plain_out[k])
        svc.append(time.perf_counter() - t0)
    plain_qps = m / sum(svc)

    def plain_at(arr):
        """The plain arm served one query at a time at the same arrival
        times: latency = arrival to the read's return, measured."""
        lat = []
        t0 = time.perf_counter()
        for (k, q), a in zip(qs[:m], arr):
            dt = a - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            plain_solve(G, ctx, absn[k], q, plain_out[k])
            lat.append((time.perf_counter() - t0 - a) * 1e3)
        return lat

    for r in rates:
        pl = plain_at(r.pop("arrivals"))
        r["plain_p50_ms"] = percentile(pl, 50)
        r["plain_p99_ms"] = percentile(pl, 99)
        r["plain_queries"] = m
    cpu = None
    if not args.no_cpu_baseline and os.path.exists(REF_BIN):
        sample = [q for k, q in qs if k != "demo"]
        kq, ref_ms = reference_full_runs(sample)
        cpu = {"value": kq / (ref_ms * 1e-3), "unit": "queries/s", "cores": 1, "kind": "reference",
               "sample": f"the first {kq} queries of the stream against the 20x20x16x10 and 32x32x24x16 models, "
                         f"each a full run of the reference's CPU method as shipped (one thread): {ref_ms:.0f} ms "
                         f"by its own timers; the 65x65x38x25 model's queries are left out of the sample (its "
                         f"abstraction alone takes about two minutes on one core), which favours the CPU"}
    line = {
        "metric": "served queries/s", "value": X, "unit": "queries/s", "n_gpus": 1, "steps": 1,
        "warmup": len(warm), "ms_per_step": sat_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 bit-sliced sets / int32 counts (f64 boxes)", "data": "synthetic",
        "config": {"workload": f"served_{n}_queries_3_models_seed{args.seed}",
                   "models": {k: models[k]["name"] for k in names}, "queries": n,
                   "budget_gb": args.serve_budget_gb, "result_buffers_in_flight": depth,
                   "sat_warp_tasks": args.sat_warp_tasks,
                   "iterations_per_step": st_ips},
        "saturation": {"throughput_qps": X, "p50_ms": percentile(sat_lat, 50), "p99_ms": percentile(sat_lat, 99)},
        "rates": rates,
        "e2e": {"value": X, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(11 * S[k] for k, _ in qs)),
                "note": "submit to results in pinned host memory, all queries"},
        "plain_sequential": {"throughput_qps": plain_qps, "queries_timed": m,
                             "p50_service_ms": percentile([x * 1e3 for x in svc], 50),
                             "p99_service_ms": percentile([x * 1e3 for x in svc], 99)},
        "speedup_vs_plain": X / plain_qps,
        "cpu_baseline": cpu,
        "server": st,
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))
    for a in absn.values():
        a.close()
    ctx.close()


def bench_simulate(args):
    """Closed-loop simulation of the published demo's controller
    (postprocess_controller.py's workload, scaled out): `--trajectories`
    seeded start states, `--sim-steps` sample periods of 32 Euler substeps.
    value = trajectories/s of gsc_problem_simulate returning final states and
    stop steps (start states in, summaries out, inside the timed call); e2e =
    the same returning every visited state; cpu_baseline = the numpy port on
    a bounded sample."""
    import numpy as np
    import torch
    import gsc_b200 as G

    sys.path.insert(0, ORACLE)
    import sim_oracle as S

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    case = C.hyperbolic_demo_case()
    ctx = G.Context(0)
    absn = G.Abstraction(ctx, case)
    prob = G.Problem(ctx, absn, case, G.METHOD_FUSED)
    prob.solve(graph=True)
    n, steps, K = args.trajectories, args.sim_steps, int(case["integration_substeps"])
    rng = np.random.default_rng(args.seed)
    x0 = rng.uniform([-1.8, -1.8, -3.1, 0.1], [1.8, 1.8, 3.1, 1.9], (n, 4))
    for _ in range(args.warmup):
        prob.simulate(x0[: 1 << 14], steps, 1, trajectories=False)
    times = []
    with ClockSampler(gpu_uuid(torch, dev)) as clocks:
        for k in range(args.steps):
            t0 = time.perf_counter()
            r = prob.simulate(x0, steps, 1000 + k, trajectories=False)
            times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    substeps = int(r["steps_done"].astype(np.int64).sum()) * K
    m = min(n, 1 << 16)
    e2e = []
    for k in range(3):
        t0 = time.perf_counter()
        prob.simulate(x0[:m], steps, 2000 + k, trajectories=True)
        e2e.append(time.perf_counter() - t0)
    te = statistics.median(e2e)
    ctl = prob.read()["controller"]
    shape, ishape = C.grid_shape(case)
    ms = 512
    t0 = time.perf_counter()
    S.simulate(ctl, S.grid_of(case, shape, ishape), x0[:ms], steps, 3)
    tc = time.perf_counter() - t0
    line = {
        "metric": "controller simulation trajectories/s", "value": n / t, "unit": "trajectories/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"simulate_hyperbolic_demo_{n}_trajectories_{steps}_periods",
                   "trajectories": n, "periods": steps, "substeps_per_period": K,
                   "substeps_simulated": substeps, "substeps_per_s": substeps / t,
                   "mean_periods_before_stop": float(r["steps_done"].mean())},
        "e2e": {"value": m / te, "unit": "trajectories/s", "h2d_bytes_per_step": 32 * m,
                "d2h_bytes_per_step": m * (steps + 1) * 32 + 36 * m, "ms_per_step": te * 1e3,
                "note": f"{m} trajectories with every visited state returned"},
        "cpu_baseline": {"value": ms / tc, "unit": "trajectories/s", "cores": 1, "kind": "port",
                         "sample": f"{ms} of the same start states through oracle/sim_oracle.py (numpy, vectorised)"},
        # one k_simulate launch per device chunk of (256 MB / 68 B) trajectories
        "gpu_launches": args.steps * -(-n // min(n, (256 << 20) // 68)),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))
    prob.close()
    absn.close()
    ctx.close()


def bench_sharded(args, case):
    """One problem solved by all ranks together (strong scaling): every rank
    owns a contiguous range of (theta, v) slices, and each iteration
    all-gathers D' over NCCL and sums two counts (gsc_shard).  One step = one
    whole sharded fixpoint; its time is the max over ranks of the device-
    synchronised wall time of the loop (the loop synchronises with the host
    every iteration)."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    import gsc_b200 as G
    import gsc_shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29533")
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    ctx = G.Context(local)
    absn = G.Abstraction(ctx, case)
    prob = G.Problem(ctx, absn, case, G.METHOD_FUSED)
    comm = gsc_shard.TorchComm(dist)
    shape, ishape = G.grid_shape(case)
    P = int(np.prod(shape)) * ishape[0] * ishape[1]
    times, res = [], None
    for k in range(args.warmup + args.steps):
        dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = gsc_shard.ShardedFixpoint(gsc_shard.DeviceEngine(prob), comm).run()
        torch.cuda.synchronize(dev)
        if k >= args.warmup:
            times.append((time.perf_counter() - t0) * 1e3)
    ms = max_over_ranks(dist, [statistics.mean(times)], dev)[0]
    one = None
    if rank == 0:
        prob.solve(graph=True)
        one = prob.read()
        same = all(np.array_equal(res[k], one[k]) for k in ("reachable_mask", "controller", "reach_step"))
        line = {
            "metric": "fixpoint pair-checks/s", "value": P * res["iterations"] / (ms * 1e-3), "unit": "pair-checks/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u32 bit-sliced sets / int32 counts (f64 boxes)", "data": "synthetic",
            "config": {"workload": case["name"], "pairs": P, "iterations": res["iterations"],
                       "parallelism": f"slice shards x{world}, NCCL all-gather of D' per iteration",
                       "same_as_one_gpu_solve": bool(same)},
        }
        print(json.dumps(line))
    prob.close()
    absn.close()
    ctx.close()
    dist.destroy_process_group()


def main():
    args = parse()
    if args.workload in ("batched", "served", "simulate") and args.impl != "reference":
        {"batched": bench_batched, "served": bench_served, "simulate": bench_simulate}[args.workload](args)
        return
    if args.workload in ("batched", "served", "simulate"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched, served or "
                                                              "device simulation mode"}))
        return
    case = C.checked(C.PRESETS[args.workload]())
    if args.impl == "reference":
        run_reference_arm(args, case)
        return
    if args.shard:
        bench_sharded(args, case)
        return

    import numpy as np
    import torch
    import gsc_b200 as G

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    method = {"auto": G.METHOD_AUTO, "stored": G.METHOD_STORED, "fused": G.METHOD_FUSED}[args.method]

    ctx = G.Context(local, stream.cuda_stream)
    absn = G.Abstraction(ctx, case)
    prob = G.Problem(ctx, absn, case, method)
    shape, ishape = G.grid_shape(case)
    S = int(np.prod(shape))
    M = ishape[0] * ishape[1]
    P = S * M

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2
    for _ in range(args.warmup):
        flush.fill_(1)
        prob.solve(graph=True)
    torch.cuda.synchronize(dev)
    iters = prob.timings()["iterations"]

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(uuid) as clocks:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            evs[k][0].record(stream)
            prob.solve(graph=True)
            evs[k][1].record(stream)
            launches += prob.timings()["kernel_launches"]
        torch.cuda.synchronize(dev)
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(dist, [sum(step_ms)], dev)[0]
    ms_per_step = total_ms / args.steps
    value = replica_value(world, P * iters, ms_per_step)

    # Dominant kernel: one profiled solve (events around each satisfaction launch).
    prob.solve(profile=True)
    tp = prob.timings()
    ph = prob.phase_timings()
    nit = max(ph["profiled_iterations"], 1)
    phases = {"prefix_or_dilation_us": 1e3 * ph["prefix_build_total_ms"] / nit,
              "pass_us": [1e3 * v / nit for v in ph["scan_axis_ms"] if v > 0],
              "satisfaction_us": 1e3 * ph["pair_satisfaction_ms"] / nit,
              "finalize_or_control_us": 1e3 * ph["reduce_inputs_ms"] / nit,
              "note": "per iteration of one host-loop solve, its launches queued behind a short hold so that they "
                      "run back to back, with CUDA events between the phases (each event adds about 2.5 us)"}
    used = tp["method"]
    kname = "k_sat_stored" if used == G.METHOD_STORED else "k_sat_col"
    per_launch_ms = tp["sat_kernel_ms"] / max(tp["sat_launches"], 1)
    alg = algorithmic_bytes(used, {"shape": shape}, tp)
    peak, peak_kind = measured_peak()
    achieved = alg / (per_launch_ms * 1e-3) / 1e9
    traffic = ncu_traffic(kname, case["name"])
    issue = issue_roofline(kname, case["name"], per_launch_ms, clocks.summary().get("sm_mhz"),
                           torch.cuda.get_device_properties(dev).multi_processor_count)

    # End to end through the public one-shot call: host description in, pinned host arrays out.
    e2e_ms = []
    pin = {k: torch.empty(S * sz, dtype=torch.uint8, pin_memory=True)
           for k, sz in (("valid_mask", 1), ("candidate_mask", 1), ("reachable_mask", 1), ("controller", 4),
                         ("reach_step", 4))}
    outs = {k: (v.numpy() if k.endswith("mask") else v.numpy().view(np.uint32)) for k, v in pin.items()}
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        # A one-shot call iterates from the host loop: a CUDA graph's
        # instantiation (about 0.3 ms) is not repaid by one solve.
        r = G.run_case(case, method=method, graph=False, device=local, out=outs)
        torch.cuda.synchronize(dev)
        if k > 0:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = max_over_ranks(dist, [statistics.median(e2e_ms)], dev)[0]
    K = case["integration_substeps"]
    h2d = 8 * (2 * shape[2] * ishape[1] * K + shape[3] * ishape[0] * K + shape[2] * ishape[1] +
               shape[3] * ishape[0]) + 64 * len(case.get("obstacles", []))
    d2h = 11 * S + 16 * r["iterations"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_BIN):
        threads = cpu_threads()
        rb = reference_bench(case, threads, 0, 1, single=False)
        st = rb["steps"][0]
        cpu = {"value": S * M / (st["step_ms"] * 1e-3), "unit": "pair-checks/s", "cores": threads,
               "kind": "reference",
               "sample": f"one full-grid fixpoint iteration of the same workload through the reference's own CPU "
                         f"method (prefix build + every state's body, reachability.hpp:53-109), states split over "
                         f"{threads} threads: {st['step_ms']:.0f} ms; the abstraction built once before it, untimed"}
    refgpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        refgpu = reference_gpu_beside_ours(G, torch, dev, stream)

    vs = None
    if args.workload == "hyperbolic_demo":
        vs = value / (PUBLISHED_DEMO_PAIRS * 12 / (PUBLISHED_DEMO_SOLVE_MS * 1e-3))
    line = {
        "metric": "fixpoint pair-checks/s", "value": value, "unit": "pair-checks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": vs, "dtype": "u32 bit-sliced sets / int32 counts (f64 boxes)",
        "data": "synthetic",
        "config": {"workload": case["name"], "states": S, "inputs": M, "pairs": P, "iterations": iters,
                   "method": {1: "stored", 2: "fused"}[used], "fixpoint_ms": ms_per_step,
                   "l2": "flushed before every step (256 MiB write)", "wall_s": t_wall,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": kname,
                     "kernel_ms_per_launch": per_launch_ms, "algorithmic_bytes_per_launch": alg,
                     "peak_kind": peak_kind, "issue": issue},
        "cpu_baseline": cpu,
        "e2e": {"value": replica_value(world, P * r["iterations"], e2e_step), "unit": "pair-checks/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step},
        "phases": phases,
        "pair_tests": {"per_step": tp["pair_tests"], "per_s": tp["pair_tests"] / (ms_per_step * 1e-3),
                       "note": "(state, input) tests the kernels actually performed per fixpoint; the rest of the "
                               "nominal pair-checks were skipped exactly (states already decided, inputs after the "
                               "first satisfied one, boxes with no cell that left the set)"},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if refgpu is not None:
        line["reference_gpu"] = refgpu
    if rank == 0:
        print(json.dumps(line))
    prob.close()
    absn.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
