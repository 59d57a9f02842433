"""Adaptive-CFL Burgers stepping on the device (solver_1d.py:148-179).

The reference loops in Python with a ``max_u.item()`` host round trip per
substep.  Here one launch runs the whole substep loop: the global max |u|,
dt_local = min(remaining, CFL dx / max|u|), the Euler substep and the
1000-substep cap all happen on the GPU, so ``step`` never synchronises."""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as nat
from .solvers import _check_state, _contig

MAX_SUBSTEPS = 1000  # solver_1d.py:155


def burgers_step_adaptive(solver, u):
    _check_state(u, solver.resolution)
    if solver.time_scheme != "euler":
        raise ValueError("adaptive_CFL sub-steps with forward Euler, as the reference does")
    u = u.contiguous()
    launch = solver.launch_for(u)
    s = _contig(solver.correction_s)
    if torch.is_grad_enabled() and (u.requires_grad or (s is not None and s.requires_grad)):
        raise NotImplementedError("gradients through adaptive_CFL stepping are not provided; use a fixed dt")
    out = torch.empty_like(u)
    rows = u.shape[0]
    t_out = torch.empty(rows, device=u.device, dtype=torch.float32)
    subs = torch.zeros(1, device=u.device, dtype=torch.int32)
    with torch.cuda.device(u.device):
        rc = nat.lib().inc_burgers_step_adaptive(
            C.byref(launch.desc), float(solver.adaptive_CFL), MAX_SUBSTEPS, u.data_ptr(), nat.ptr(s),
            nat.ptr(launch.t_rows), launch.t0, out.data_ptr(), t_out.data_ptr(), None, subs.data_ptr(),
            nat.stream_of(u.device))
    nat.check(rc, "inc_burgers_step_adaptive")
    # self.t advances by the sub-step sum, which equals dt unless the cap stopped early
    if isinstance(solver.t, torch.Tensor):
        solver.t.copy_(t_out.reshape(solver.t.shape).to(solver.t.dtype))
    else:
        solver._t_dev = t_out
        solver.t = solver.t + solver.dt
    solver._substeps_dev = subs
    if solver.LOG is not None:
        solver.LOG.info(f"CFL: {solver.adaptive_CFL}, using substeps: {int(subs.item())}, time_step: {solver.dt}")
    return out
