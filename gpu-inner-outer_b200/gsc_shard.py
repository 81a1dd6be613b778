"""Sharded fixpoint: one K-invariance problem solved by several ranks.

The reference solves a case on one GPU (cuda/kernels.cu:654-767 loops over
every state each iteration).  Here G ranks -- one process per GPU, or threads
of one process for ranks that share a device -- each hold the whole problem
and iterate only their own contiguous range of (theta, v) slices.  States are
x-fastest, so a slice range is one contiguous slab of every state array and
of the bit-sliced D' = (valid and not reachable) or unsafe.

One iteration on every rank (the Jacobi update of reachability.hpp:53-109):

1. ``engine.step()``: the (theta, v) dilation of D' over the whole grid, then
   the satisfaction test, the exists-input reduction and the finalize of the
   rank's own slices; returns its newly reachable and newly certified counts.
2. ``comm.exchange_dprime``: an all-gather of the ranks' D' slabs, so every
   rank holds the whole next D' (S / 8 bytes in all: 0.5 MB at 65x65x38x25).
3. ``comm.sum``: an all-reduce of the two counts.
4. ``engine.control(nr, nc)``: the reference's stop rules
   (reachability.hpp:133-144) with the summed counts, alike on every rank.

After the stop every rank gathers the slabs of the result arrays
(``comm.gather_slabs``), so each returns the whole result.

Engines: ``DeviceEngine`` drives a ``gsc_b200.Problem`` through the C ABI's
``gsc_problem_shard_*`` entry points.  Comms: ``TorchComm`` over a
``torch.distributed`` process group (NCCL all-gathers D' in device memory;
other backends stage it through host memory), ``ThreadComm`` for ranks that
are threads of one process.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

import gsc_b200 as G


def partition(slices: int, world: int):
    """Contiguous near-equal slice ranges: rank r owns [lo_r, hi_r)."""
    if world < 1 or slices < world:
        raise ValueError(f"cannot split {slices} slices over {world} ranks")
    return [(slices * r // world, slices * (r + 1) // world) for r in range(world)]


RESULT_SLABS = ("valid_mask", "candidate_mask", "reachable_mask", "controller", "reach_step")


class ShardedFixpoint:
    """Runs one engine's share of a sharded solve in lockstep with the other
    ranks of ``comm``; ``run()`` returns the whole result on every rank."""

    def __init__(self, engine, comm):
        self.engine = engine
        self.comm = comm

    def run(self) -> dict:
        eng, comm = self.engine, self.comm
        ranges = partition(eng.slices, comm.world)
        lo, hi = ranges[comm.rank]
        eng.begin(lo, hi)
        iterations = 0
        while True:
            nr, nc = eng.step()
            comm.exchange_dprime(eng, ranges)
            eng.sync()
            nr, nc = comm.sum([nr, nc])
            iterations += 1
            if eng.control(nr, nc):
                break
            if iterations > eng.iteration_bound:
                raise RuntimeError("sharded fixpoint did not stop within its iteration bound")
        res = eng.read()
        per_slice = eng.states_per_slice
        bounds = [(a * per_slice, b * per_slice) for a, b in ranges]
        for key in RESULT_SLABS:
            res[key] = comm.gather_slabs(res[key], bounds)
        res["shard"] = {"rank": comm.rank, "world": comm.world, "slices": (lo, hi)}
        return res


class DeviceEngine:
    """One rank's share of a sharded solve on its GPU (gsc_problem_shard_*)."""

    def __init__(self, problem: "G.Problem"):
        self.p = problem
        r = problem.read(masks=False)
        n0, n1, n2, n3 = (int(v) for v in r["shape"])
        self.slices = n2 * n3
        self.states_per_slice = n0 * n1
        self.iteration_bound = int(r["states"]) + 2
        ptr = ctypes.c_void_p()
        wps = ctypes.c_uint64()
        problem.ctx.check(G.lib().gsc_problem_shard_words(problem._h, ctypes.byref(ptr), ctypes.byref(wps)))
        self.words_per_slice = int(wps.value)
        self._dp_ptr = int(ptr.value)
        self._dp = None

    def dprime(self):
        """The problem's D' words as a torch tensor (int32 view of device memory)."""
        if self._dp is None:
            import torch

            n = self.slices * self.words_per_slice

            class _View:
                __cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (self._dp_ptr, False),
                                            "version": 3}

            self._dp = torch.as_tensor(_View(), device=torch.device("cuda", self.p.ctx.device))
        return self._dp

    def begin(self, lo, hi):
        self.p.ctx.check(G.lib().gsc_problem_shard_begin(self.p._h, int(lo), int(hi)))

    def sync(self):
        """Waits for the exchange's writes into D' (made on torch's streams)
        before the library's next launch on its own stream."""
        import torch

        torch.cuda.synchronize(torch.device("cuda", self.p.ctx.device))

    def step(self):
        c = (ctypes.c_uint64 * 2)()
        self.p.ctx.check(G.lib().gsc_problem_shard_step(self.p._h, c))
        return int(c[0]), int(c[1])

    def control(self, nr, nc) -> bool:
        stop = ctypes.c_int()
        self.p.ctx.check(G.lib().gsc_problem_shard_control(self.p._h, int(nr), int(nc), ctypes.byref(stop)))
        return bool(stop.value)

    def read(self) -> dict:
        return self.p.read()

    # host staging of D' slabs (for comms without device collectives)
    def dprime_slab_host(self, lo, hi):
        w = self.words_per_slice
        return self.dprime()[lo * w:hi * w].cpu().numpy()

    def set_dprime_slab_host(self, lo, hi, words):
        import torch

        w = self.words_per_slice
        self.dprime()[lo * w:hi * w].copy_(torch.from_numpy(np.ascontiguousarray(words)))


class TorchComm:
    """Collectives of one rank over a torch.distributed process group.  With
    the NCCL backend D' is all-gathered in device memory (over NVLink between
    GPUs); with others it is staged through host memory."""

    def __init__(self, dist):
        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.nccl = dist.get_backend() == "nccl"

    def sum(self, values):
        import torch

        dev = torch.device("cuda", torch.cuda.current_device()) if self.nccl else torch.device("cpu")
        t = torch.tensor([int(v) for v in values], dtype=torch.int64, device=dev)
        self.dist.all_reduce(t)
        return [int(v) for v in t.tolist()]

    def exchange_dprime(self, engine, ranges):
        import torch

        w = engine.words_per_slice
        most = max(hi - lo for lo, hi in ranges) * w
        lo, hi = ranges[self.rank]
        if self.nccl:
            dp = engine.dprime()
            send = torch.zeros(most, dtype=torch.int32, device=dp.device)
            send[:(hi - lo) * w] = dp[lo * w:hi * w]
            recv = torch.empty(self.world * most, dtype=torch.int32, device=dp.device)
            self.dist.all_gather_into_tensor(recv, send)
            for r, (a, b) in enumerate(ranges):
                if r != self.rank:
                    dp[a * w:b * w] = recv[r * most:r * most + (b - a) * w]
            return
        send = torch.zeros(most, dtype=torch.int32)
        send[:(hi - lo) * w] = torch.from_numpy(engine.dprime_slab_host(lo, hi))
        parts = [torch.empty(most, dtype=torch.int32) for _ in range(self.world)]
        self.dist.all_gather(parts, send)
        for r, (a, b) in enumerate(ranges):
            if r != self.rank:
                engine.set_dprime_slab_host(a, b, parts[r][:(b - a) * w].numpy())

    def gather_slabs(self, arr, bounds):
        """Every rank's own slab [lo, hi) of a state array, assembled on every rank."""
        import torch

        arr = np.ascontiguousarray(arr)
        raw = arr.view(np.uint8)
        isz = arr.dtype.itemsize
        most = max(hi - lo for lo, hi in bounds) * isz
        lo, hi = bounds[self.rank]
        dev = torch.device("cuda", torch.cuda.current_device()) if self.nccl else torch.device("cpu")
        send = torch.zeros(most, dtype=torch.uint8, device=dev)
        send[:(hi - lo) * isz] = torch.from_numpy(raw[lo * isz:hi * isz]).to(dev)
        parts = [torch.empty(most, dtype=torch.uint8, device=dev) for _ in range(self.world)]
        self.dist.all_gather(parts, send)
        out = raw.copy()
        for r, (a, b) in enumerate(bounds):
            out[a * isz:b * isz] = parts[r][:(b - a) * isz].cpu().numpy()
        return out.view(arr.dtype)


class ThreadComm:
    """Collectives between ranks that are threads of one process (``world``
    threads share one ThreadComm through ``for_rank``).  Each collective is a
    barrier round: ranks post their part, wait for all, read the others'."""

    def __init__(self, world):
        self.world = world
        self._bar = threading.Barrier(world)
        self._slots = [None] * world

    def for_rank(self, rank):
        outer = self

        class _Rank:
            def __init__(self):
                self.rank = rank
                self.world = outer.world

            def _round(self, value):
                outer._slots[rank] = value
                outer._bar.wait()
                got = list(outer._slots)
                outer._bar.wait()
                return got

            def sum(self, values):
                got = self._round([int(v) for v in values])
                return [sum(g[i] for g in got) for i in range(len(values))]

            def exchange_dprime(self, engine, ranges):
                lo, hi = ranges[rank]
                w = engine.words_per_slice
                mine = engine.dprime()[lo * w:hi * w].clone()
                got = self._round(mine)
                for r, (a, b) in enumerate(ranges):
                    if r != rank:
                        engine.dprime()[a * w:b * w].copy_(got[r].to(engine.dprime().device))

            def gather_slabs(self, arr, bounds):
                got = self._round(np.ascontiguousarray(arr))
                out = np.array(arr, copy=True)
                for r, (a, b) in enumerate(bounds):
                    out[a:b] = got[r][a:b]
                return out

        return _Rank()


def solve_threads(case, world: int, device: int = 0) -> dict:
    """The sharded solve with `world` ranks as threads of this process on one
    device, each rank with its own context (stream), abstraction and problem,
    as separate processes would hold them.  Returns rank 0's (whole) result."""
    comm = ThreadComm(world)
    out, errs = [None] * world, []

    def body(r):
        ctx = absn = prob = None
        try:
            ctx = G.Context(device)
            absn = G.Abstraction(ctx, case)
            prob = G.Problem(ctx, absn, case, G.METHOD_FUSED)
            out[r] = ShardedFixpoint(DeviceEngine(prob), comm.for_rank(r)).run()
        except Exception as e:   # noqa: BLE001
            errs.append(e)
            comm._bar.abort()
        finally:
            for h in (prob, absn, ctx):
                if h is not None:
                    h.close()

    ths = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    if errs:
        raise errs[0]
    return out[0]
