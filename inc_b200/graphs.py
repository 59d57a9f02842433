"""CUDA-graph replay of corrector-in-the-loop rollouts.

``GraphedRollout`` records the loop of ``simulate_rollout`` (trainer/trainer_1d.py:154-183:
``s = model(u); solver.correction_s = s; u = solver.step(u); results[:, k] = u``) for a
fixed batch shape once, as one CUDA graph, and replays it for new initial states:
every step's corrector kernels (torch) and solver launch (this library) run without
host round trips or per-launch overhead.  Evaluation only (no autograd graph).  This
is for corrector shapes the fused kernels do not cover (for example the FNO with the
KS solver); for the periodic CNN with Burgers, ``simulate_rollout`` already runs the
corrector inside the solver kernel.

The launches are recorded with the solver's time at capture (``solver.t``, which a
Burgers ``"learning"`` forcing source reads), so every replay starts from that time;
after a replay ``solver.t`` reads capture time + steps * dt, and
``solver.correction_s`` the last correction, as after ``simulate_rollout``.
Construct a new ``GraphedRollout`` to start from another time.
"""
from __future__ import annotations

import torch

from .solvers import BurgersSolverTorch, KSSolverTorch


class GraphedRollout:
    def __init__(self, model, solver, u_example: torch.Tensor, steps: int, domain_size=None,
                 corrections: bool = True, warmup: int = 2):
        if not isinstance(solver, (BurgersSolverTorch, KSSolverTorch)):
            raise TypeError("GraphedRollout: solver must be a BurgersSolverTorch or KSSolverTorch")
        if isinstance(solver, BurgersSolverTorch) and solver.adaptive_CFL is not None:
            raise ValueError("GraphedRollout: adaptive_CFL solvers choose their substeps on the device each "
                             "call; capture needs a fixed dt")
        if not u_example.is_cuda:
            raise ValueError("GraphedRollout: u_example must be a CUDA tensor")
        self.model, self.solver, self.steps = model, solver, int(steps)
        self.domain_size = domain_size
        dev = u_example.device
        B, N = u_example.shape
        self.u_in = torch.empty(B, N, device=dev, dtype=torch.float32)
        self.u_in.copy_(u_example)
        self.frames = torch.empty(B, self.steps, N, device=dev, dtype=torch.float32)
        self.corr = torch.empty_like(self.frames) if corrections else None
        self._t0 = solver.t.clone() if isinstance(getattr(solver, "t", None), torch.Tensor) else \
            getattr(solver, "t", None)
        if isinstance(solver, KSSolverTorch):
            solver.plan_for(self.u_in, domain_size)  # the plan's one-time upload happens outside capture
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.no_grad(), torch.cuda.stream(side):
            for _ in range(max(1, warmup)):
                self._reset_time()
                self._loop()
        torch.cuda.current_stream(dev).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        self._reset_time()
        with torch.no_grad(), torch.cuda.graph(self.graph):
            self._loop()
        self._reset_time()

    def _reset_time(self):
        if self._t0 is not None:
            self.solver.t = self._t0.clone() if isinstance(self._t0, torch.Tensor) else self._t0

    def _loop(self):
        u = self.u_in
        L = self.domain_size
        for k in range(self.steps):
            s = self.model(u) if L is None else self.model(u, L)
            self.solver.correction_s = s
            u = self.solver.step(u) if L is None else self.solver.step(u, L)
            self.frames[:, k].copy_(u)
            if self.corr is not None:
                self.corr[:, k].copy_(s)

    def __call__(self, u0: torch.Tensor):
        """(frames [B, steps, N], corrections or None) for initial state u0 (same shape
        as at capture).  The returned tensors are the graph's buffers: the next call
        overwrites them."""
        if u0.shape != self.u_in.shape:
            raise ValueError(f"GraphedRollout: u0 shape {tuple(u0.shape)} != captured {tuple(self.u_in.shape)}")
        self.u_in.copy_(u0)
        self.graph.replay()
        if self._t0 is not None:  # the recorded launches start at the capture time
            self.solver.t = self._t0 + self.steps * self.solver.dt
        if self.corr is not None:
            self.solver.correction_s = self.corr[:, -1]
        return self.frames, self.corr
