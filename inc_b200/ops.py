"""Single operators of the reference exposed on the GPU."""
from __future__ import annotations

import torch

from . import _native as nat


def weno_reconstruction(f: torch.Tensor, direction: str = "left") -> torch.Tensor:
    """WENO5 reconstruction of each periodic row of f; solver_1d.py:4-42.

    'left' gives f+ at i+1/2 from f[i-2..i+2]; 'right' gives the reference's
    right-biased value from f[i-1..i+3].  f: [rows, n] FP32 CUDA, n a power of
    two in [8, 512]."""
    if direction not in ("left", "right"):
        raise ValueError("Direction must be 'left' or 'right'.")
    if not f.is_cuda or f.dtype != torch.float32 or f.dim() != 2:
        raise ValueError("f must be a [rows, n] float32 CUDA tensor")
    f = f.contiguous()
    out = torch.empty_like(f)
    if f.shape[0] == 0:  # no rows: nothing to launch
        return out
    with torch.cuda.device(f.device):
        rc = nat.lib().inc_weno_reconstruct(f.data_ptr(), out.data_ptr(), f.shape[0], f.shape[1],
                                            0 if direction == "left" else 1, nat.stream_of(f.device))
    nat.check(rc, "inc_weno_reconstruct")
    return out
