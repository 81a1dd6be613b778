"""A CPU stand-in for gsc_shard.DeviceEngine, for the multi-rank tests
(test infrastructure only).  It runs one rank's share of a sharded solve with
the oracle's per-state iteration (orc_spot_step: iteration k of
reachability.hpp:53-109 for listed states, from the whole previous state)
and applies the reference's stop rules (reachability.hpp:133-144) on the
host.  What it exchanges between ranks in place of D' is its slab of the
reachable set, one int32 word per state, which is all the next iteration's
test needs from the other ranks."""
import numpy as np

import oracle as O

INVALID = 0xFFFFFFFF
MESSAGES = {1: "all candidate states obtained a controller", 2: "iteration stalled before candidate closure",
            3: "maximum iterations reached"}


class OracleShardEngine:
    def __init__(self, case):
        self.case = case
        start = O.solve(dict(case, max_iterations=0))
        n0, n1, n2, n3 = (int(v) for v in start["shape"])
        self.slices = n2 * n3
        self.states_per_slice = n0 * n1
        self.words_per_slice = n0 * n1
        self.S = n0 * n1 * n2 * n3
        self.iteration_bound = self.S + 2
        self.valid = start["valid_mask"]
        self.cand = start["candidate_mask"]
        self.max_iterations = int(case["max_iterations"])

    def begin(self, lo, hi):
        self.lo, self.hi = lo * self.states_per_slice, hi * self.states_per_slice
        self.reach = self.cand.astype(np.int32)
        self.ctl = np.full(self.S, INVALID, np.uint32)
        self.step_ = np.where(self.cand != 0, 0, INVALID).astype(np.uint32)
        self.iter = 0
        self.candidates = int(self.cand.sum())
        self.certified = 0
        self.reachable = self.candidates
        self.stopped = self.max_iterations == 0
        self.message = 3 if self.stopped else 0
        self.new_reachable, self.new_certified = [], []

    def step(self):
        if self.stopped:
            return 0, 0
        states = np.arange(self.lo, self.hi, dtype=np.uint64)
        reach8 = self.reach.astype(np.uint8)
        rn, ct, st = O.spot_step(self.case, self.valid, self.cand, reach8, self.ctl, self.step_, self.iter + 1,
                                 states)
        own = slice(self.lo, self.hi)
        nr = int(np.count_nonzero((rn != 0) & (reach8[own] == 0)))
        nc = int(np.count_nonzero((self.cand[own] != 0) & (self.ctl[own] == INVALID) & (ct != INVALID)))
        self.reach[own] = rn
        self.ctl[own] = ct
        self.step_[own] = st
        return nr, nc

    def sync(self):
        pass

    def dprime_slab_host(self, lo, hi):
        w = self.words_per_slice
        return self.reach[lo * w:hi * w].copy()

    def set_dprime_slab_host(self, lo, hi, words):
        w = self.words_per_slice
        self.reach[lo * w:hi * w] = words

    def control(self, nr, nc):
        if self.stopped:
            return True
        self.iter += 1
        self.certified += nc
        self.reachable += nr
        self.new_reachable.append(nr)
        self.new_certified.append(nc)
        if self.certified == self.candidates:
            self.message, self.stopped = 1, True
        elif nr == 0 and nc == 0:
            self.message, self.stopped = 2, True
        elif self.iter >= self.max_iterations:
            self.message, self.stopped = 3, True
        return self.stopped

    def read(self):
        return {"valid_mask": self.valid.copy(), "candidate_mask": self.cand.copy(),
                "reachable_mask": self.reach.astype(np.uint8), "controller": self.ctl.copy(),
                "reach_step": self.step_.copy(), "iterations": self.iter, "message": MESSAGES[self.message],
                "reachable_states": self.reachable, "certified_candidates": self.certified,
                "iter_new_reachable": np.array(self.new_reachable, np.uint64),
                "iter_new_certified": np.array(self.new_certified, np.uint64)}
