"""Hybrid rollouts with the corrector evaluated inside the solver kernel.

``burgers_cnn_rollout`` runs the loop of ``simulate_rollout``
(trainer/trainer_1d.py:154-183: ``s = model(u); solver.correction_s = s;
u = solver.step(u); results[:, k] = u``) for a ``PeriodicCNN1D`` corrector in
one launch of ``inc_burgers_cnn_rollout``: the four convolutions run from
shared memory before every step, so no per-step corrector launches remain.
Forward only -- evaluation rollouts under ``torch.no_grad()``; training keeps
the per-step graph (torch corrector plus the CUDA solver's autograd
functions).  ``simulate_rollout`` dispatches here by itself when gradients are
off and the model and solver qualify (``cnn_supported``).
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
            and u.shape[1] in CNN_N and u.shape[1] == solver.resolution)


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


def burgers_cnn_rollout(model, solver, u0, steps, corrections=True):
    """(frames [B, steps, N], corrections [B, steps, N] or None) of the hybrid rollout,
    as ``simulate_rollout(model, solver, u0, steps, "INC")`` computes them.

    Advances ``solver.t`` by steps * dt and leaves the last correction in
    ``solver.correction_s``, like the per-step loop."""
    if not cnn_supported(model, solver, u0):
        raise ValueError("burgers_cnn_rollout: needs a PeriodicCNN1D(32, 5, 4) corrector, a fixed-dt "
                         "BurgersSolverTorch and a CUDA float32 state of width 64, 128, 256 or 512")
    u0 = u0.detach().contiguous()
    steps = int(steps)
    launch = solver.launch_for(u0)
    w = pack_cnn_weights(model, u0.device)
    B, N = u0.shape
    frames = torch.empty(B, steps, N, device=u0.device, dtype=torch.float32)
    corr = torch.empty_like(frames) if corrections else None
    launch.cnn_rollout(w, u0, steps, frames, corr, None)
    solver.t += steps * solver.dt
    solver.correction_s = corr[:, -1] if (corr is not None and steps > 0) else None
    return frames, corr
