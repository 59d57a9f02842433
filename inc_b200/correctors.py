"""Corrector networks s(u) for the hybrid rollouts (torch modules).

The corrector stays in torch; the solver step around it is the CUDA path.
Two architectures from the benchmark configurations:

* ``PeriodicCNN1D`` - 4 circular Conv1d layers (32 channels, kernel 5) with
  GELU between them: [B, N] -> [B, N].
* ``FNO1D`` - a Fourier neural operator (Li et al., 2021): lift (u, x/L grid)
  to `width` channels, 4 layers of spectral convolution (keep the lowest
  `modes` rFFT modes, complex weights) plus a 1x1 convolution, GELU between
  layers, project with two linear layers.  ``forward(u, L)`` takes the
  per-trajectory domain size like the reference's FNO corrector
  (models/models_1d/fno.py:39-105) does.
"""
from __future__ import annotations

import torch
import torch.nn as nn
import torch.nn.functional as F


class PeriodicCNN1D(nn.Module):
    def __init__(self, channels: int = 32, kernel: int = 5, layers: int = 4):
        super().__init__()
        widths = [1] + [channels] * (layers - 1) + [1]
        self.convs = nn.ModuleList(
            nn.Conv1d(widths[i], widths[i + 1], kernel, padding=kernel // 2, padding_mode="circular")
            for i in range(layers))

    def forward(self, u, L=None):
        x = u.unsqueeze(1)
        for i, conv in enumerate(self.convs):
            x = conv(x)
            if i + 1 < len(self.convs):
                x = F.gelu(x)
        return x.squeeze(1)


class SpectralConv1d(nn.Module):
    """Multiply the lowest `modes` rFFT modes by learned complex in x out matrices."""

    def __init__(self, cin: int, cout: int, modes: int):
        super().__init__()
        self.modes = modes
        scale = 1.0 / (cin * cout)
        self.w_re = nn.Parameter(scale * torch.rand(cin, cout, modes))
        self.w_im = nn.Parameter(scale * torch.rand(cin, cout, modes))

    def forward(self, x):
        n = x.shape[-1]
        xf = torch.fft.rfft(x)
        m = min(self.modes, xf.shape[-1])
        w = torch.complex(self.w_re[..., :m], self.w_im[..., :m])
        out = torch.zeros(x.shape[0], w.shape[1], xf.shape[-1], dtype=xf.dtype, device=x.device)
        out[..., :m] = torch.einsum("bim,iom->bom", xf[..., :m], w)
        return torch.fft.irfft(out, n=n)


def _pointwise(conv: nn.Conv1d, x):
    """A kernel-size-1 Conv1d as a channel matmul (same parameters and result):
    cuDNN's FP32 weight gradient for 1x1 convolutions is a slow direct kernel,
    while the matmul's runs on cuBLAS."""
    return torch.matmul(conv.weight[:, :, 0], x) + conv.bias[:, None]


class FNO1D(nn.Module):
    def __init__(self, modes: int = 16, width: int = 64, layers: int = 4):
        super().__init__()
        self.lift = nn.Linear(2, width)
        self.spectral = nn.ModuleList(SpectralConv1d(width, width, modes) for _ in range(layers))
        self.pointwise = nn.ModuleList(nn.Conv1d(width, width, 1) for _ in range(layers))
        self.proj1 = nn.Linear(width, 128)
        self.proj2 = nn.Linear(128, 1)

    def forward(self, u, L=None):
        B, n = u.shape
        base = torch.linspace(0, 1, n, dtype=u.dtype, device=u.device)
        if L is None:
            grid = base.expand(B, n)
        elif isinstance(L, torch.Tensor):
            grid = L.reshape(B, 1).to(u.dtype) * base
        else:
            grid = float(L) * base.expand(B, n)
        x = self.lift(torch.stack([u, grid], dim=-1)).permute(0, 2, 1)
        for i, (sc, pw) in enumerate(zip(self.spectral, self.pointwise)):
            x = sc(x) + _pointwise(pw, x)
            if i + 1 < len(self.spectral):
                x = F.gelu(x)
        x = F.gelu(self.proj1(x.permute(0, 2, 1)))
        return self.proj2(x).squeeze(-1)
