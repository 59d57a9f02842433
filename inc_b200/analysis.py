"""Post-rollout analysis on the GPU."""
from __future__ import annotations

import math

import torch

from . import _native as nat


def energy_spectrum(velocity: torch.Tensor):
    """Energy spectrum of every frame, on the GPU (analysis/Plot_KS.py:196-235).

    velocity: [B, T, D] or [T, D] FP32 CUDA tensor, D a power of two in
    [16, 512].  Returns (energy [B, T, D//2+1], k_phys [B, D//2+1]) with
    energy[..., k] = |FFT(u)[k]|^2, bins 1..D/2-1 doubled, k_phys = 2 pi k."""
    if velocity.dim() == 2:
        velocity = velocity.unsqueeze(0)
    if velocity.dim() != 3 or not velocity.is_cuda or velocity.dtype != torch.float32:
        raise ValueError("velocity must be a [B, T, D] (or [T, D]) float32 CUDA tensor")
    B, T, D = velocity.shape
    v = velocity.contiguous()
    out = torch.empty(B, T, D // 2 + 1, device=v.device, dtype=torch.float32)
    with torch.cuda.device(v.device):
        rc = nat.lib().inc_energy_spectrum(v.data_ptr(), out.data_ptr(), B * T, D, nat.stream_of(v.device))
    nat.check(rc, "inc_energy_spectrum")
    k = 2 * math.pi * torch.arange(D // 2 + 1, device=v.device, dtype=torch.float32)
    return out, k.expand(B, -1).contiguous()
