"""Restatement of the reference's trajectory windowing (test infrastructure only).

data/data_loader_1d.py:8-118 of tum-pbs/INC: a [B, T+1, D] trajectory tensor
is cut into (u_initial, u_target[mstep]) windows that start every
`starts_gap` frames and step `n_substeps = round(dt / gen_dt)` frames."""
import numpy as np


def windows(trajectories, gen_dt, dt, mstep, starts_gap):
    traj = np.asarray(trajectories)
    ratio = dt / gen_dt
    if abs(ratio - round(ratio)) > 1e-6:
        raise ValueError(f"dt must be a multiple of gen_dt ({gen_dt})")
    nsub = int(round(ratio))
    total = traj.shape[1] - 1
    starts = np.arange(0, total - nsub * mstep + 1, starts_gap)
    items = []
    for idx in range(traj.shape[0] * len(starts)):
        b, s = idx // len(starts), starts[idx % len(starts)]
        seg = traj[b, s:s + nsub * mstep + 1:nsub]
        items.append((b, int(s), seg[0], seg[1:]))
    return items
