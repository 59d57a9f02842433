"""Adaptive-CFL Burgers stepping on the device (solver_1d.py:148-179).

The reference loops in Python with a ``max_u.item()`` host round trip per
substep.  Here one cooperative launch over all SMs runs the whole substep loop:
the global max |u|, dt_local = min(remaining, CFL dx / max|u|), the Euler
substep and the 1000-substep stop all happen on the GPU, so ``step`` never
synchronises.

Gradients: as autograd through the reference, where dt_local comes from
``.item()`` and is a constant, the backward differentiates the substeps that ran
with their recorded sizes (``inc_burgers_step_adaptive_bwd``).  It reads the
substep count from the device once (to size its scratch), so a backward through
an adaptive step synchronises there, where the reference's forward synchronised
once per substep."""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as nat
from .solvers import _check_state, _contig

MAX_SUBSTEPS = 1000  # solver_1d.py:155
_ERR_OFFSET, _RUN_OFFSET = 20, 24  # int32 fields of the work buffer's control block


def _work(device):
    n = int(nat.lib().inc_burgers_step_adaptive_work_size(MAX_SUBSTEPS))
    return torch.empty(n, dtype=torch.uint8, device=device)


def run_info(work):
    """(substeps run, error flag) of the adaptive step recorded in `work` (a host sync)."""
    v = work[:32].view(torch.int32).cpu()
    return int(v[_RUN_OFFSET // 4]), int(v[_ERR_OFFSET // 4])


class AdaptiveStepFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, s, launch, cfl, t_out, subs):
        out = torch.empty_like(u)
        work = _work(u.device)
        with nat.on_device(u.device):
            rc = nat.lib().inc_burgers_step_adaptive(
                C.byref(launch.desc), float(cfl), MAX_SUBSTEPS, u.data_ptr(), nat.ptr(s), nat.ptr(launch.t_rows),
                launch.t0, out.data_ptr(), t_out.data_ptr(), work.data_ptr(), subs.data_ptr(),
                nat.stream_of(u.device))
        nat.check(rc, "inc_burgers_step_adaptive")
        ctx.launch, ctx.has_s = launch, s is not None
        ctx.save_for_backward(u, s if s is not None else u.new_empty(0), work)
        return out

    @staticmethod
    def backward(ctx, g):
        u, s, work = ctx.saved_tensors
        s = s if ctx.has_s else None
        executed, err = run_info(work)
        if err:
            raise RuntimeError(f"adaptive step recorded error {err}; its gradient is not defined")
        gu = torch.empty_like(u)
        gs = torch.empty_like(u) if (ctx.has_s and ctx.needs_input_grad[1]) else None
        states = torch.empty(max(executed, 1), *u.shape, device=u.device, dtype=u.dtype)
        launch = ctx.launch
        with nat.on_device(u.device):
            rc = nat.lib().inc_burgers_step_adaptive_bwd(
                C.byref(launch.desc), u.data_ptr(), nat.ptr(s), nat.ptr(launch.t_rows), launch.t0, work.data_ptr(),
                MAX_SUBSTEPS, executed, g.contiguous().data_ptr(), gu.data_ptr(), nat.ptr(gs), states.data_ptr(),
                nat.stream_of(u.device))
        nat.check(rc, "inc_burgers_step_adaptive_bwd")
        return gu, gs, None, None, None, None


def burgers_step_adaptive(solver, u):
    _check_state(u, solver.resolution)
    if solver.time_scheme != "euler":
        raise ValueError("adaptive_CFL sub-steps with forward Euler, as the reference does")
    u = u.contiguous()
    launch = solver.launch_for(u)
    s = _contig(solver.correction_s)
    if s is not None:
        _check_state(s, solver.resolution, "correction_s")
    rows = u.shape[0]
    # the step's start time for every row (the forcing source reads it; t_out is built on it
    # whatever the equation type)
    launch._bind_time(solver.t, rows)
    t_out = torch.empty(rows, device=u.device, dtype=torch.float32)
    subs = torch.zeros(1, device=u.device, dtype=torch.int32)
    out = AdaptiveStepFn.apply(u, s, launch, solver.adaptive_CFL, t_out, subs)
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
