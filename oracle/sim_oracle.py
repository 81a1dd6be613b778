"""CPU restatement of the controller's closed-loop simulation -- TEST
INFRASTRUCTURE ONLY (the checker of gsc_problem_simulate; never shipped or
measured).

Follows plots/postprocess_controller.py of the reference:
  * state_to_flat_index (:66-101): theta wrapped with atan2(sin, cos) on a
    copy, index = round((x - lb) / eta) per dimension (round half to even),
    clamped to [0, n - 1], flattened x-fastest;
  * get_control_input (:103-130): controller lookup, stop at the invalid
    input, input centre of the flat input index j = i_a + m_a * i_omega;
  * update_state (:132-176): x + dt * (f(x, u) + w) per element, theta
    wrapped with atan2(sin, cos);
  * simulate_trajectory (:178-224): `steps` sample periods of
    `integration_substeps` Euler substeps, a uniform disturbance in
    [-dhw, dhw] per dimension and substep, rows after a stop left at zero.

The reference draws its disturbances from numpy's global generator; here
(and on the device) they come from Philox4x32-10 (Salmon, Moraes, Dror and
Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011) keyed by the
seed, with counter (2 * (step * K + substep) + half, trajectory, 0, 0): each
call gives two doubles of 53 random bits ((a >> 5) * 2^26 + (b >> 6)) / 2^53,
mapped like numpy's uniform, low + (high - low) * u.
"""
from __future__ import annotations

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32 with 10 rounds; arguments are uint64 arrays (or
    scalars) holding 32-bit values."""
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & MASK for v in (c0, c1, c2, c3))
    k0 = np.uint64(k0 & MASK)
    k1 = np.uint64(k1 & MASK)
    for _ in range(10):
        p0 = np.uint64(M0) * c0
        p1 = np.uint64(M1) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(MASK)
        hi1, lo1 = p1 >> np.uint64(32), p1 & np.uint64(MASK)
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & np.uint64(MASK), lo1, (hi0 ^ c3 ^ k1) & np.uint64(MASK), lo0
        k0 = (k0 + np.uint64(W0)) & np.uint64(MASK)
        k1 = (k1 + np.uint64(W1)) & np.uint64(MASK)
    return c0, c1, c2, c3


def u53(a, b):
    return ((a >> np.uint64(5)).astype(np.float64) * 67108864.0 + (b >> np.uint64(6)).astype(np.float64)) \
        / 9007199254740992.0


def disturbances(seed: int, traj, step: int, substep: int, K: int, dhw):
    """The four disturbance components of one substep for trajectories `traj`."""
    traj = np.asarray(traj, dtype=np.uint64)
    base = 2 * (step * K + substep)
    k0, k1 = seed & MASK, (seed >> 32) & MASK
    u = []
    for half in (0, 1):
        r = philox4x32_10(np.full(traj.shape, base + half, np.uint64), traj, 0, 0, k0, k1)
        u.append(u53(r[0], r[1]))
        u.append(u53(r[2], r[3]))
    dhw = np.asarray(dhw, dtype=np.float64)
    low, high = -dhw, dhw
    return np.stack([low[d] + (high[d] - low[d]) * u[d] for d in range(4)], axis=-1)


def grid_of(case, shape, input_shape):
    """The simulation's grid parameters of a case dict."""
    return {"state_lb": case["state_lb"], "state_eta": case["state_eta"], "shape": list(shape),
            "input_lb": case["input_lb"], "input_eta": case["input_eta"], "input_shape": list(input_shape),
            "sample_time": case["sample_time"], "integration_substeps": case["integration_substeps"],
            "disturbance_half_width": case["disturbance_half_width"]}


def flat_index(state, lb, eta, shape):
    """postprocess_controller.py:66-101 for rows of states."""
    s = np.array(state, dtype=np.float64, copy=True)
    s[..., 2] = np.arctan2(np.sin(s[..., 2]), np.cos(s[..., 2]))
    idx = np.round((s - lb) / eta).astype(np.int64)
    idx = np.clip(idx, 0, np.asarray(shape, dtype=np.int64) - 1)
    strides = np.array([1, shape[0], shape[0] * shape[1], shape[0] * shape[1] * shape[2]], dtype=np.int64)
    return (idx * strides).sum(axis=-1)


def simulate(controller, grid, x0, steps: int, seed: int, ids=None):
    """grid: dict with state_lb, state_eta, shape, input_lb, input_eta,
    input_shape, sample_time, integration_substeps, disturbance_half_width.
    ids: the trajectories' indices in the RNG counter (default 0 .. n-1).
    Returns (trajectories [n][steps+1][4], steps_done [n])."""
    x0 = np.asarray(x0, dtype=np.float64).reshape(-1, 4)
    n = x0.shape[0]
    lb = np.asarray(grid["state_lb"], np.float64)
    eta = np.asarray(grid["state_eta"], np.float64)
    shape = [int(v) for v in grid["shape"]]
    ilb = np.asarray(grid["input_lb"], np.float64)
    ieta = np.asarray(grid["input_eta"], np.float64)
    ma, mw = (int(v) for v in grid["input_shape"])
    K = int(grid["integration_substeps"])
    dt = float(grid["sample_time"]) / K
    dhw = grid["disturbance_half_width"]
    traj = np.zeros((n, steps + 1, 4))
    traj[:, 0] = x0
    done = np.zeros(n, np.uint32)
    alive = np.ones(n, bool)
    x = x0.copy()
    ids = np.arange(n) if ids is None else np.asarray(ids)
    for step in range(steps):
        j = controller[flat_index(x, lb, eta, shape)].astype(np.int64)
        ok = alive & (j != 0xFFFFFFFF) & (j < ma * mw)
        alive = ok
        if not alive.any():
            break
        a = ilb[0] + (j % ma + 0.5) * ieta[0]
        w = ilb[1] + (j // ma + 0.5) * ieta[1]
        for sub in range(K):
            d = disturbances(seed, ids, step, sub, K, dhw)
            f = np.stack([x[:, 3] * np.cos(x[:, 2]), x[:, 3] * np.sin(x[:, 2]), w, a], axis=-1)
            xn = x + dt * (f + d)
            xn[:, 2] = np.arctan2(np.sin(xn[:, 2]), np.cos(xn[:, 2]))
            x = np.where(alive[:, None], xn, x)
        traj[alive, step + 1] = x[alive]
        done[alive] += 1
    return traj, done
