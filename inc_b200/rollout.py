"""Fused multi-step rollouts and the ``simulate_rollout`` drop-in.

``simulate_rollout`` keeps the signature and return value of
``trainer/trainer_1d.py:154-183`` (tum-pbs/INC).  Without a corrector network
(``correction_term=None``) the whole rollout is one kernel launch with the state
held on chip; with one (``"INC"``) the network runs in torch between single
solver steps, as in the reference, optionally under ``torch.utils.checkpoint``
every ``checkpoint_every`` steps.

``burgers_rollout`` / ``ks_rollout`` are differentiable: their backward replays
``ckpt_every``-step segments from checkpoints stored by the forward launch and
runs the hand-written adjoint kernels on them.
"""
from __future__ import annotations

import torch
import torch.utils.checkpoint as tuc

from .solvers import BurgersSolverTorch, KSSolverTorch, _check_state, _contig


def _nseg(steps, k):
    return (steps + k - 1) // k


class BurgersRolloutFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, s, launch, steps, ckpt_every, want_grad):
        B, N = u0.shape
        frames = torch.empty(B, steps, N, device=u0.device, dtype=u0.dtype)
        ckpts = torch.empty(B, _nseg(steps, ckpt_every), N, device=u0.device, dtype=u0.dtype) if want_grad else None
        launch.rollout(u0, s, steps, frames, None, ckpt_every, ckpts)
        ctx.launch, ctx.steps, ctx.k, ctx.has_s = launch, steps, ckpt_every, s is not None
        if want_grad:
            ctx.save_for_backward(ckpts, s if s is not None else u0.new_empty(0))
        return frames

    @staticmethod
    def backward(ctx, g_frames):
        ckpts, s = ctx.saved_tensors
        s = s if ctx.has_s else None
        g_u0 = torch.empty(ckpts.shape[0], ckpts.shape[2], device=ckpts.device, dtype=ckpts.dtype)
        g_s = torch.empty_like(g_u0) if (ctx.has_s and ctx.needs_input_grad[1]) else None
        ctx.launch.rollout_bwd(ckpts, s, ctx.steps, ctx.k, g_frames.contiguous(), None, g_u0, g_s)
        return g_u0, g_s, None, None, None, None


class KSRolloutFn(torch.autograd.Function):
    """ckpt_every > 0: checkpoints every ckpt_every steps, segments replayed in the
    backward; ckpt_every == 0: a tape of every step's states (no replay, more memory)."""

    @staticmethod
    def forward(ctx, u0, s, plan, steps, ckpt_every, want_grad):
        B, N = u0.shape
        frames = torch.empty(B, steps, N, device=u0.device, dtype=u0.dtype)
        if want_grad and ckpt_every == 0:
            saved = torch.empty(plan.tape_size(steps), dtype=torch.uint8, device=u0.device)
            plan.rollout_tape(u0, s, steps, frames, None, saved)
        else:
            k = ckpt_every if ckpt_every > 0 else 8
            saved = torch.empty(B, _nseg(steps, k), N, device=u0.device, dtype=u0.dtype) if want_grad else None
            plan.rollout(u0, s, steps, frames, None, k, saved)
        ctx.plan, ctx.steps, ctx.k, ctx.has_s = plan, steps, ckpt_every, s is not None
        ctx.shape = (B, N)
        if want_grad:
            ctx.save_for_backward(saved, s if s is not None else u0.new_empty(0))
        return frames

    @staticmethod
    def backward(ctx, g_frames):
        saved, s = ctx.saved_tensors
        s = s if ctx.has_s else None
        g_u0 = torch.empty(ctx.shape, device=saved.device, dtype=torch.float32)
        g_s = torch.empty_like(g_u0) if (ctx.has_s and ctx.needs_input_grad[1]) else None
        if ctx.k == 0:
            ctx.plan.rollout_bwd_tape(saved, s, ctx.steps, g_frames.contiguous(), None, g_u0, g_s)
        else:
            ctx.plan.rollout_bwd(saved, s, ctx.steps, ctx.k, g_frames.contiguous(), None, g_u0, g_s)
        return g_u0, g_s, None, None, None, None


def burgers_rollout(solver: BurgersSolverTorch, u0, steps, s=None, ckpt_every=8):
    """Frames [B, steps, N] of `steps` fixed steps in one launch (s held constant).

    Differentiable w.r.t. u0 and s.  Advances ``solver.t`` by steps * dt."""
    if solver.adaptive_CFL is not None:
        raise ValueError("fused rollouts use a fixed dt; adaptive_CFL solvers step one call at a time")
    _check_state(u0, solver.resolution)
    u0 = u0.contiguous()
    launch = solver.launch_for(u0) if u0.shape[0] else None
    s = _contig(s)
    if s is not None:
        _check_state(s, solver.resolution, "s")
    want = torch.is_grad_enabled() and (u0.requires_grad or (s is not None and s.requires_grad))
    if u0.shape[0] == 0:  # an empty batch: nothing to launch
        frames = u0.unsqueeze(1).expand(0, int(steps), u0.shape[1]).clone()
    else:
        frames = BurgersRolloutFn.apply(u0, s, launch, int(steps), int(ckpt_every), want)
    solver.t += steps * solver.dt
    return frames


def ks_rollout(solver: KSSolverTorch, u0, steps, domain_size, s=None, ckpt_every=8):
    """Frames [B, steps, N] of `steps` KS step() calls in one launch (s held constant).

    Differentiable w.r.t. u0 and s.  The backward replays ckpt_every-step segments from
    checkpoints; ckpt_every=0 records every step's states in a tape instead (32 bytes per
    row pair, cell and step) and the backward reads them, with no replay."""
    _check_state(u0, solver.resolution)
    u0 = u0.contiguous()
    s = _contig(s)
    if s is not None:
        _check_state(s, solver.resolution, "s")
    if u0.shape[0] == 0:  # an empty batch: nothing to launch
        return u0.unsqueeze(1).expand(0, int(steps), u0.shape[1]).clone()
    plan = solver.plan_for(u0, domain_size)
    want = torch.is_grad_enabled() and (u0.requires_grad or (s is not None and s.requires_grad))
    return KSRolloutFn.apply(u0, s, plan, int(steps), int(ckpt_every), want)


def simulate_rollout(model, solver, u_initial, mstep, correction_term, L=None, checkpoint_every=None):
    """Drop-in for trainer/trainer_1d.py:154-183.

    Returns (results [B, mstep, D], corrections [B, mstep, D] or None)."""
    B, D = u_initial.shape
    solver.correction_s = None
    if correction_term is None:
        if isinstance(solver, KSSolverTorch) and solver.correction_u is None:
            return ks_rollout(solver, u_initial, mstep, L), None
        if isinstance(solver, BurgersSolverTorch) and solver.adaptive_CFL is None:
            return burgers_rollout(solver, u_initial, mstep), None
    elif correction_term != "INC":
        raise ValueError(f"Invalid correction term: {correction_term}")
    else:
        from . import fused
        if not torch.is_grad_enabled():
            if fused.cnn_supported(model, solver, u_initial):  # evaluation: corrector inside the solver kernel
                return fused.burgers_cnn_rollout(model, solver, u_initial, mstep)
        elif fused.cnn_train_supported(model, solver, u_initial):  # training: fused forward and backward
            k = int(checkpoint_every or 8)
            if 1 <= k <= fused.max_ckpt_every(u_initial.shape[1]):
                return fused.burgers_cnn_rollout(model, solver, u_initial, mstep, ckpt_every=k)

    model_fn = (lambda u: model(u)) if L is None else (lambda u: model(u, L))
    step_fn = (lambda u: solver.step(u)) if L is None else (lambda u: solver.step(u, L))

    def one(u):
        c = model_fn(u) if correction_term == "INC" else None
        solver.correction_s = c
        return step_fn(u), c

    results, corrections = [], []
    u = u_initial
    k = int(checkpoint_every or 0)
    step = 0
    while step < mstep:
        if k > 1 and torch.is_grad_enabled() and correction_term == "INC":
            span = min(k, mstep - step)
            t_save = solver.t.clone() if isinstance(getattr(solver, "t", None), torch.Tensor) else getattr(solver, "t", None)

            def segment(u_in, span=span, t_save=t_save):
                if t_save is not None:
                    solver.t = t_save.clone() if isinstance(t_save, torch.Tensor) else t_save
                outs, cs = [], []
                x = u_in
                for _ in range(span):
                    x, c = one(x)
                    outs.append(x)
                    cs.append(c)
                return tuple(outs) + tuple(cs)

            out = tuc.checkpoint(segment, u, use_reentrant=False)
            results += list(out[:span])
            corrections += list(out[span:])
            u = out[span - 1]
            step += span
        else:
            u, c = one(u)
            results.append(u)
            corrections.append(c)
            step += 1
    res = torch.stack(results, dim=1)
    cor = torch.stack(corrections, dim=1) if correction_term == "INC" else None
    return res, cor
