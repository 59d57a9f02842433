"""Hybrid rollouts with the corrector evaluated inside the solver kernel.

``burgers_cnn_rollout`` runs the loop of ``simulate_rollout``
(trainer/trainer_1d.py:154-183: ``s = model(u); solver.correction_s = s;
u = solver.step(u); results[:, k] = u``) for a ``PeriodicCNN1D`` corrector in
one launch of ``inc_burgers_cnn_rollout``: the four convolutions run from
shared memory before every step, so no per-step corrector launches remain.
With gradients on (rows of 64, 128, 256 or 512 cells), the rollout is one autograd node
whose backward is ``inc_burgers_cnn_rollout_bwd``: segment replay from
checkpoints, the network's activations recomputed in shared memory, the
solver's adjoint and the network's backward in one kernel, weight gradients
summed over rows in a fixed order.  ``simulate_rollout`` dispatches here by
itself when the model and solver qualify (``cnn_supported`` /
``cnn_train_supported``); otherwise it keeps the per-step loop.
"""
from __future__ import annotations

import torch

from . import _native as nat
from .correctors import PeriodicCNN1D

CNN_N = (64, 128, 256, 512)
_CNN_LAYERS = ((1, 32), (32, 32), (32, 32), (32, 1))


def _cnn_shape_ok(model) -> bool:
    convs = getattr(model, "convs", None)
    if convs is None or len(convs) != len(_CNN_LAYERS):
        return False
    for conv, (ci, co) in zip(convs, _CNN_LAYERS):
        if (conv.in_channels, conv.out_channels) != (ci, co) or conv.kernel_size != (5,) or conv.padding != (2,):
            return False
        if conv.padding_mode != "circular" or conv.stride != (1,) or conv.dilation != (1,) or conv.groups != 1:
            return False
        if conv.bias is None:
            return False
    return True


def cnn_supported(model, solver, u) -> bool:
    """True when the fused kernel computes exactly this model and solver on state u."""
    from .solvers import BurgersSolverTorch
    return (isinstance(model, PeriodicCNN1D) and type(model).forward is PeriodicCNN1D.forward
            and _cnn_shape_ok(model)
            and isinstance(solver, BurgersSolverTorch) and solver.adaptive_CFL is None
            and isinstance(u, torch.Tensor) and u.is_cuda and u.dtype == torch.float32 and u.dim() == 2
            and u.shape[0] > 0 and u.shape[1] in CNN_N and u.shape[1] == solver.resolution)


def pack_cnn_weights(model, device=None) -> torch.Tensor:
    """The kernel's weight layout: w1[co][k], b1, w2[ci][co][k], b2, w3[ci][co][k], b3, w4[ci][k], b4."""
    if not _cnn_shape_ok(model):
        raise ValueError("pack_cnn_weights: model is not a PeriodicCNN1D(32 channels, kernel 5, 4 layers)")
    w = [c.weight.detach().float() for c in model.convs]
    b = [c.bias.detach().float() for c in model.convs]
    parts = [w[0][:, 0, :].reshape(-1), b[0], w[1].transpose(0, 1).reshape(-1), b[1],
             w[2].transpose(0, 1).reshape(-1), b[2], w[3][0].reshape(-1), b[3]]
    out = torch.cat([p.to(device) for p in parts]).contiguous()
    if out.numel() != nat.INC_CNN_WEIGHT_FLOATS:
        raise ValueError(f"pack_cnn_weights: {out.numel()} floats, expected {nat.INC_CNN_WEIGHT_FLOATS}")
    return out


CNN_TRAIN_N = CNN_N
MAX_CKPT_EVERY = 32
# Largest record of the hidden layers' pre-activations the training path keeps (bytes):
# 2 x 32 x n floats per row and step, 537 MB for 256 rows x 256 cells x 32 steps.
ACTS_BYTES_MAX = 4 << 30


def max_ckpt_every(n: int) -> int:
    """Largest segment length of the fused backward at row width n (its segment
    states share the SM's 227 KB of shared memory with the activations)."""
    return 26 if n == 512 else MAX_CKPT_EVERY


def cnn_train_supported(model, solver, u) -> bool:
    """True when the fused training kernel (forward + backward) covers this case."""
    return cnn_supported(model, solver, u) and u.shape[1] in CNN_TRAIN_N


def unpack_cnn_grads(g: torch.Tensor):
    """Packed gradient -> (w1, b1, w2, b2, w3, b3, w4, b4) in torch's Conv1d shapes."""
    C, K = 32, 5
    o = [0]

    def take(n):
        v = g[o[0]:o[0] + n]
        o[0] += n
        return v
    w1 = take(C * K).view(C, 1, K)
    b1 = take(C)
    w2 = take(C * C * K).view(C, C, K).transpose(0, 1).contiguous()
    b2 = take(C)
    w3 = take(C * C * K).view(C, C, K).transpose(0, 1).contiguous()
    b3 = take(C)
    w4 = take(C * K).view(1, C, K)
    b4 = take(1)
    return w1, b1, w2, b2, w3, b3, w4, b4


class BurgersCNNRolloutFn(torch.autograd.Function):
    """Frames and corrections of the fused hybrid rollout, differentiable w.r.t. u0 and
    the eight parameters of the corrector."""

    @staticmethod
    def forward(ctx, u0, launch, steps, ckpt_every, *params):
        B, N = u0.shape
        w = _pack_params(params, u0.device)
        frames = torch.empty(B, steps, N, device=u0.device, dtype=torch.float32)
        corr = torch.empty_like(frames)
        nseg = (steps + ckpt_every - 1) // ckpt_every
        ckpts = torch.empty(B, nseg, N, device=u0.device, dtype=torch.float32)
        # the hidden layers' pre-activations of every step, kept for the backward when they
        # fit ACTS_BYTES_MAX (else the backward recomputes them)
        acts = None
        if B * steps * 2 * 32 * N * 4 <= ACTS_BYTES_MAX:
            acts = torch.empty(B, steps, 2, 32, N, device=u0.device, dtype=torch.float32)
        launch.cnn_rollout(w, u0, steps, frames, corr, None, ckpt_every, ckpts, acts=acts)
        ctx.save_for_backward(ckpts, corr, w, acts)
        ctx.launch, ctx.steps, ctx.ckpt_every, ctx.shape = launch, steps, ckpt_every, (B, N)
        return frames, corr

    @staticmethod
    def backward(ctx, g_frames, g_corr):
        ckpts, corr, w, acts = ctx.saved_tensors
        B, N = ctx.shape
        dev = ckpts.device
        g_u0 = torch.empty(B, N, device=dev, dtype=torch.float32)
        g_w = torch.empty(nat.INC_CNN_WEIGHT_FLOATS, device=dev, dtype=torch.float32)
        work = torch.empty(B, nat.INC_CNN_WEIGHT_FLOATS, device=dev, dtype=torch.float32)
        gf = None if g_frames is None else g_frames.contiguous()
        gc = None if g_corr is None else g_corr.contiguous()
        ctx.launch.cnn_rollout_bwd(w, ckpts, corr, ctx.steps, ctx.ckpt_every, gf, gc, None, g_u0, g_w, work,
                                   acts=acts)
        return (g_u0, None, None, None) + unpack_cnn_grads(g_w)


def _pack_params(params, device):
    w1, b1, w2, b2, w3, b3, w4, b4 = [p.detach().float() for p in params]
    out = torch.cat([w1[:, 0, :].reshape(-1), b1, w2.transpose(0, 1).reshape(-1), b2,
                     w3.transpose(0, 1).reshape(-1), b3, w4[0].reshape(-1), b4]).to(device).contiguous()
    return out


def burgers_cnn_rollout(model, solver, u0, steps, corrections=True, ckpt_every=8):
    """(frames [B, steps, N], corrections [B, steps, N] or None) of the hybrid rollout,
    as ``simulate_rollout(model, solver, u0, steps, "INC")`` computes them.

    With gradients enabled (and u0 or the model's parameters requiring them) the
    result is differentiable through the fused backward, which replays
    ckpt_every-step segments (n = 64, 128, 256 or 512).  Advances ``solver.t`` by steps * dt and
    leaves the last correction in ``solver.correction_s``, like the per-step loop."""
    if not cnn_supported(model, solver, u0):
        raise ValueError("burgers_cnn_rollout: needs a PeriodicCNN1D(32, 5, 4) corrector, a fixed-dt "
                         "BurgersSolverTorch and a CUDA float32 state of width 64, 128, 256 or 512")
    steps = int(steps)
    params = [p for c in model.convs for p in (c.weight, c.bias)]
    want = torch.is_grad_enabled() and (u0.requires_grad or any(p.requires_grad for p in params))
    if want and steps > 0:
        k, kmax = int(ckpt_every), max_ckpt_every(u0.shape[1])
        if not 1 <= k <= kmax:
            raise ValueError(f"burgers_cnn_rollout: ckpt_every must be in [1, {kmax}] for rows of "
                             f"{u0.shape[1]} cells")
        u0c = u0.contiguous()
        launch = solver.launch_for(u0c)
        frames, corr = BurgersCNNRolloutFn.apply(u0c, launch, steps, k, *params)
    else:
        u0c = u0.detach().contiguous()
        launch = solver.launch_for(u0c)
        w = pack_cnn_weights(model, u0c.device)
        B, N = u0c.shape
        frames = torch.empty(B, steps, N, device=u0c.device, dtype=torch.float32)
        corr = torch.empty_like(frames) if corrections else None
        launch.cnn_rollout(w, u0c, steps, frames, corr, None)
    solver.t += steps * solver.dt
    solver.correction_s = corr[:, -1] if (corr is not None and steps > 0) else None
    return frames, (corr if corrections else None)
