"""Training data on the GPU: trajectory generation with the fused solvers and
windowed sampling in the reference's dataset format.

The reference trains from ``INC_Data/*.pth`` dictionaries holding
``trajectories`` [B, T+1, D] plus per-trajectory parameters (``nu``, ``A``,
``omega``, ``phi``, ``l`` for Burgers, ``domain_size`` for KS) and
``metadata['gen_dt']``; ``BurgersDataset`` / ``KSDataset``
(data/data_loader_1d.py:8-118) cut them into windows and the collate
functions (:120-139) batch them.  ``TrajectoryWindows`` does the same with
index arithmetic on GPU-resident tensors (one gather per batch, no per-item
Python), and ``generate_*`` produce such dictionaries with the fused rollout
kernels (the reference's datasets are not part of this repository).
"""
from __future__ import annotations

import torch

BURGERS_KEYS = ("nu", "A", "omega", "phi", "l")


class TrajectoryWindows:
    """Windows (u_initial, u_target[mstep]) of a trajectory dictionary.

    Same indexing as the reference datasets: item i takes trajectory
    i // S at start starts[i % S], S = len(starts), starts =
    arange(0, T - n_sub * mstep + 1, starts_gap), n_sub = round(dt / gen_dt).
    ``starts_gap=None`` means n_sub (the reference's default, which it builds
    as a float and cannot index with)."""

    def __init__(self, data, dt=None, mstep=1, starts_gap=None, kind="burgers", device=None):
        self.kind = kind
        traj = data["trajectories"]
        self.device = torch.device(device) if device is not None else traj.device
        self.traj = traj.to(self.device)
        self.gen_dt = float(data["metadata"]["gen_dt"])
        self.dt = self.gen_dt if dt is None else float(dt)
        ratio = self.dt / self.gen_dt
        if abs(ratio - round(ratio)) > 1e-6:
            raise ValueError(f"dt must be a multiple of gen_dt ({self.gen_dt})")
        self.n_sub = int(round(ratio))
        gap = self.n_sub if starts_gap is None else int(starts_gap)
        total = self.traj.shape[1] - 1
        self.mstep = int(mstep)
        self.starts = torch.arange(0, total - self.n_sub * self.mstep + 1, gap, device=self.device)
        self.offsets = self.n_sub * torch.arange(self.mstep + 1, device=self.device)
        if kind == "burgers":
            self.params = {k: data[k].to(self.device) for k in BURGERS_KEYS}
        elif kind == "ks":
            self.params = {"domain_size": data["domain_size"].to(self.device)}
        else:
            raise ValueError(f"unknown kind {kind!r}")

    def __len__(self):
        return self.traj.shape[0] * len(self.starts)

    def batch(self, idx: torch.Tensor):
        """The collated batch of items `idx` (as BG_collate_fn / KS_collate_fn)."""
        idx = idx.to(self.device)
        S = len(self.starts)
        b = idx // S
        start = self.starts[idx % S]
        seg = self.traj[b[:, None], start[:, None] + self.offsets[None, :]]  # [n, mstep+1, D]
        out = {"u_initial": seg[:, 0], "u_target": seg[:, 1:]}
        if self.kind == "burgers":
            for k, v in self.params.items():
                out[k] = v[b]
            out["t"] = start.to(self.traj.dtype) * self.gen_dt
        else:
            out["domain_size"] = self.params["domain_size"][b].reshape(-1)
        return out

    def loader(self, batch_size, shuffle=False, generator=None):
        n = len(self)
        order = torch.randperm(n, generator=generator) if shuffle else torch.arange(n)
        for i in range(0, n, batch_size):
            yield self.batch(order[i:i + batch_size])


def generate_ks(solver, u0, domain_size, steps, s=None):
    """A KS trajectory dictionary from the fused rollout: [B, steps+1, D] frames
    (u0 first) spaced by one solver step (2 dt), the reference's data format."""
    from .rollout import ks_rollout
    with torch.no_grad():
        frames = ks_rollout(solver, u0, steps, domain_size, s=s)
    traj = torch.cat([u0.unsqueeze(1), frames], dim=1)
    return {"trajectories": traj, "domain_size": domain_size.reshape(-1, 1).clone(),
            "metadata": {"gen_dt": 2 * float(solver.dt), "resolution": solver.resolution}}


def generate_burgers(solver, u0, steps):
    """A Burgers trajectory dictionary from the fused rollout (forcing parameters
    and nu taken from the solver's sim_params)."""
    from .rollout import burgers_rollout
    p = solver.param
    t0 = solver.t
    with torch.no_grad():
        frames = burgers_rollout(solver, u0, steps)
    traj = torch.cat([u0.unsqueeze(1), frames], dim=1)
    B = u0.shape[0]
    out = {"trajectories": traj, "metadata": {"gen_dt": float(solver.dt), "resolution": solver.resolution,
                                              "L": float(solver.L), "t0": t0}}
    nu = solver.nu
    out["nu"] = (nu.reshape(B, 1).clone() if isinstance(nu, torch.Tensor)
                 else torch.full((B, 1), float(nu), device=u0.device))
    for k in ("A", "omega", "phi", "l"):
        v = getattr(p, k, None)
        if v is not None:
            out[k] = torch.as_tensor(v, device=u0.device).reshape(B, 1, -1).clone()
    return out
