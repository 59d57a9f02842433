"""Corrector networks s(u) for the hybrid rollouts (torch modules).

Two architectures from the benchmark configurations:

* ``PeriodicCNN1D`` - 4 circular Conv1d layers (32 channels, kernel 5) with
  GELU between them: [B, N] -> [B, N].
* ``FNO1D`` - a Fourier neural operator (Li et al., 2021): lift (u, x/L grid)
  to `width` channels, 4 layers of spectral convolution (keep the lowest
  `modes` rFFT modes, complex weights) plus a 1x1 convolution, GELU between
  layers, project with two linear layers.  ``forward(u, L)`` takes the
  per-trajectory domain size like the reference's FNO corrector
  (models/models_1d/fno.py:39-105) does.

On CUDA tensors each FNO layer's ``spectral(x) + W x + b`` runs through
``inc_spectral_conv1d`` with a hand-written adjoint.  Its kernels are streaming
row-pair FFTs to the kept modes, the mode mixing, and streaming inverse FFTs that
add the 1x1 branch and its bias.  The projection's bias and GELU are one kernel
(``inc_bias_gelu``).  The other layers are batched matmuls (cuBLAS) on the
[B, width, n] state.  Shapes the kernels do not cover, and CPU tensors,
take torch's FFTs.  The CNN runs inside the Burgers solver kernel when
``simulate_rollout`` can fuse it (``fused.py``).
"""
from __future__ import annotations

import torch
import torch.nn as nn
import torch.nn.functional as F

from . import _native as nat


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


SPECTRAL_CONV_N = (16, 32, 64, 128, 256, 512)


def spectral_conv1d_torch(x, w_re, w_im, modes: int):
    """SpectralConv1d.forward with torch FFTs (models/models_1d/fno.py:26-37):
    rfft, the lowest `modes` modes times complex [cin][cout][modes] weights,
    irfft back to x's length."""
    n = x.shape[-1]
    xf = torch.fft.rfft(x)
    m = min(modes, xf.shape[-1])
    w = torch.complex(w_re[..., :m], w_im[..., :m])
    out = torch.zeros(x.shape[0], w.shape[1], xf.shape[-1], dtype=xf.dtype, device=x.device)
    out[..., :m] = torch.einsum("bim,iom->bom", xf[..., :m], w)
    return torch.fft.irfft(out, n=n)


def spectral_conv_supported(x, w_re, w_im, modes: int) -> bool:
    """True when ``inc_spectral_conv1d`` computes this call: FP32 CUDA tensors,
    x [B, W, n] with n a power of two in [16, 512], square weights of even width
    <= 128, 1 <= modes <= min(32, n / 2)."""
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dim() == 3 and x.dtype == torch.float32):
        return False
    B, W, n = x.shape
    return (w_re.dtype == torch.float32 and w_im.dtype == torch.float32 and w_re.is_cuda
            and tuple(w_re.shape[:2]) == (W, W) and w_im.shape == w_re.shape and W % 2 == 0 and W <= 128
            and n in SPECTRAL_CONV_N and 1 <= modes <= min(32, n // 2, w_re.shape[-1]) and B > 0)


def _spectral_work(B: int, W: int, modes: int, device):
    """Scratch of inc_spectral_conv1d: the mixed modes and the mode-major weights."""
    return torch.empty(2 * modes * W * (B + W), device=device, dtype=torch.float32)


class SpectralConv1dFn(torch.autograd.Function):
    """``inc_spectral_conv1d`` forward (with the optional bias and addend of the
    layer sum); ``inc_spectral_conv1d_bwd`` for the input gradient.  The weight
    gradient is sum_b dL/dout[b][o][k] conj(rfft(x)[b][c][k]) as one complex
    batched matmul over the modes; the bias gradient, sum over b and n of dL/dy,
    is n times the real part of the backward's DC coefficient summed over b."""

    @staticmethod
    def forward(ctx, x, w_re, w_im, bias, addend, modes: int):
        x = x.contiguous()
        wr = w_re[..., :modes].contiguous()
        wi = w_im[..., :modes].contiguous()
        B, W, n = x.shape
        if addend is not None:
            addend = addend.contiguous()
        y = torch.empty_like(x)
        need_w = ctx.needs_input_grad[1] or ctx.needs_input_grad[2]
        xm = torch.empty(B, W, modes, 2, device=x.device, dtype=torch.float32)  # rfft(x) modes
        work = _spectral_work(B, W, modes, x.device)
        rc = nat.lib().inc_spectral_conv1d(x.data_ptr(), wr.data_ptr(), wi.data_ptr(), nat.ptr(bias),
                                           nat.ptr(addend), y.data_ptr(), xm.data_ptr(), work.data_ptr(),
                                           B, W, n, modes, nat.stream_of(x.device))
        nat.check(rc, "inc_spectral_conv1d")
        ctx.save_for_backward(wr, wi, xm if need_w else None)
        ctx.modes, ctx.full_modes = modes, w_re.shape[-1]
        ctx.has_bias, ctx.has_addend = bias is not None, addend is not None
        return y

    @staticmethod
    def backward(ctx, gy):
        wr, wi, xm = ctx.saved_tensors
        gy = gy.contiguous()
        B, W, n = gy.shape
        m = ctx.modes
        need_w = ctx.needs_input_grad[1] or ctx.needs_input_grad[2]
        need_b = ctx.has_bias and ctx.needs_input_grad[3]
        gx = torch.empty_like(gy)
        gm = torch.empty(B, W, m, 2, device=gy.device, dtype=torch.float32)  # dL/dF modes
        work = _spectral_work(B, W, m, gy.device)
        rc = nat.lib().inc_spectral_conv1d_bwd(gy.data_ptr(), wr.data_ptr(), wi.data_ptr(), gx.data_ptr(),
                                               gm.data_ptr(), work.data_ptr(), B, W, n, m,
                                               nat.stream_of(gy.device))
        nat.check(rc, "inc_spectral_conv1d_bwd")
        gw_re = gw_im = g_bias = None
        if need_w:
            gw = torch.einsum("bok,bck->cok", torch.view_as_complex(gm), torch.view_as_complex(xm).conj())
            gw_re = gw.real.new_zeros(W, W, ctx.full_modes)
            gw_im = torch.zeros_like(gw_re)
            gw_re[..., :m] = gw.real
            gw_im[..., :m] = gw.imag
        if need_b:
            g_bias = gm[:, :, 0, 0].sum(0) * n
        g_add = gy if (ctx.has_addend and ctx.needs_input_grad[4]) else None
        return (gx if ctx.needs_input_grad[0] else None), gw_re, gw_im, g_bias, g_add, None


def spectral_conv1d(x, w_re, w_im, modes: int, bias=None, addend=None):
    """SpectralConv1d.forward, plus bias[:, None] and addend where given (the FNO
    layer's sum with its 1x1 convolution): the CUDA kernel where it applies,
    else torch FFTs."""
    m = min(modes, x.shape[-1] // 2 + 1)
    bias_ok = bias is None or (bias.is_cuda and bias.dtype == torch.float32 and bias.shape == x.shape[1:2])
    addend_ok = addend is None or (addend.is_cuda and addend.dtype == torch.float32 and addend.shape == x.shape)
    if spectral_conv_supported(x, w_re, w_im, m) and bias_ok and addend_ok:
        return SpectralConv1dFn.apply(x, w_re, w_im, bias, addend, m)
    y = spectral_conv1d_torch(x, w_re, w_im, modes)
    if bias is not None:
        y = y + bias[:, None]
    if addend is not None:
        y = y + addend
    return y


class SpectralConv1d(nn.Module):
    """Multiply the lowest `modes` rFFT modes by learned complex in x out matrices."""

    def __init__(self, cin: int, cout: int, modes: int):
        super().__init__()
        self.modes = modes
        scale = 1.0 / (cin * cout)
        self.w_re = nn.Parameter(scale * torch.rand(cin, cout, modes))
        self.w_im = nn.Parameter(scale * torch.rand(cin, cout, modes))

    def forward(self, x):
        return spectral_conv1d(x, self.w_re, self.w_im, self.modes)


def _channel_mm(w, x):
    """w [out, in] applied to every trajectory of x [B, in, n] -> [B, out, n] as
    one batched matmul.  (torch.matmul of a 2-D by a 3-D operand folds the batch
    into the columns, which transposes x and the result through copies, and
    makes the weight gradient one GEMM with K = B * n and a tiny output tile;
    the batched form needs neither.)  The FNO's kernel-size-1 Conv1d layers run
    as this product too (same parameters and result): cuDNN's FP32 weight
    gradient for 1x1 convolutions is a slow direct kernel."""
    return torch.bmm(w.expand(x.shape[0], -1, -1), x)


class BiasGeluFn(torch.autograd.Function):
    """gelu(h + bias[:, None]) for h [B, C, n] on CUDA: ``inc_bias_gelu`` (one pass), and
    ``inc_bias_gelu_bwd`` (gelu' and the per-row sums that give the bias gradient)."""

    @staticmethod
    def forward(ctx, h, bias):
        h = h.contiguous()
        B, C, n = h.shape
        y = torch.empty_like(h)
        rc = nat.lib().inc_bias_gelu(h.data_ptr(), bias.data_ptr(), y.data_ptr(), B * C, n, C,
                                     nat.stream_of(h.device))
        nat.check(rc, "inc_bias_gelu")
        ctx.save_for_backward(h, bias)
        return y

    @staticmethod
    def backward(ctx, gy):
        h, bias = ctx.saved_tensors
        gy = gy.contiguous()
        B, C, n = h.shape
        gh = torch.empty_like(h)
        sums = torch.empty(B * C, device=h.device, dtype=torch.float32)
        rc = nat.lib().inc_bias_gelu_bwd(gy.data_ptr(), h.data_ptr(), bias.data_ptr(), gh.data_ptr(),
                                         sums.data_ptr(), B * C, n, C, nat.stream_of(h.device))
        nat.check(rc, "inc_bias_gelu_bwd")
        return gh, sums.view(B, C).sum(0)


def bias_gelu(h, bias):
    """F.gelu(h + bias[:, None]) for h [B, C, n]: one CUDA kernel where it applies."""
    if (h.is_cuda and h.dim() == 3 and h.dtype == torch.float32 and h.shape[-1] % 4 == 0 and h.shape[0] > 0
            and isinstance(bias, torch.Tensor) and bias.is_cuda and bias.dtype == torch.float32
            and tuple(bias.shape) == (h.shape[1],)):
        return BiasGeluFn.apply(h, bias)
    return F.gelu(h + bias[:, None])


def _channel_linear(lin: nn.Linear, x):
    """nn.Linear over the channel axis of x [B, in, n] -> [B, out, n]."""
    return _channel_mm(lin.weight, x) + lin.bias[:, None]


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
        # The hidden state stays [B, width, n] (contiguous) from the lift to the
        # projection: the Linear layers act on the channel axis as channel matmuls
        # (same parameters, same result), so no permuted view reaches an
        # elementwise kernel or a gradient.
        x = _channel_linear(self.lift, torch.stack([u, grid], dim=1))
        for i, (sc, pw) in enumerate(zip(self.spectral, self.pointwise)):
            # sc(x) + pw(x) with pw's bias and product added in the spectral kernel's epilogue
            x = spectral_conv1d(x, sc.w_re, sc.w_im, sc.modes, bias=pw.bias,
                                addend=_channel_mm(pw.weight[:, :, 0], x))
            if i + 1 < len(self.spectral):
                x = F.gelu(x)
        x = bias_gelu(_channel_mm(self.proj1.weight, x), self.proj1.bias)
        return _channel_linear(self.proj2, x).squeeze(1)
