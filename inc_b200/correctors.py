"""Corrector networks s(u) for the hybrid rollouts (torch modules).

Two architectures from the benchmark configurations:

* ``PeriodicCNN1D`` - 4 circular Conv1d layers (32 channels, kernel 5) with
  GELU between them: [B, N] -> [B, N].
* ``FNO1D`` - the reference's FNO corrector (models/models_1d/fno.py:39-105):
  the same constructor ``FNO1D(L=16, modes=16, width=64)``, submodules and
  parameter names (fc0, conv0..3 with complex ``weights1``, w0..3, fc1, fc2), so
  a reference state_dict loads unchanged, and the same ``forward(u, L=None)``
  with the grid of ``get_grid`` (models/models_1d/utils.py:3-31).

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
    """The reference's Fourier layer (models/models_1d/fno.py:6-37), same constructor
    and parameter: ``weights1`` [in, out, modes1] complex64, drawn as
    scale * (U[0,1) + i U[0,1)) with scale = 1 / (in * out), so its state_dict loads
    unchanged.  forward(x [B, in, n]) -> [B, out, n]: rfft, the lowest modes1 modes
    mixed by weights1, irfft; on CUDA through ``inc_spectral_conv1d``."""

    def __init__(self, in_channels: int, out_channels: int, modes1: int):
        super().__init__()
        self.in_channels = in_channels
        self.out_channels = out_channels
        self.modes1 = modes1
        self.scale = 1 / (in_channels * out_channels)
        self.weights1 = nn.Parameter(self.scale * torch.rand(in_channels, out_channels, modes1, dtype=torch.cfloat))

    def weights_re_im(self, dtype):
        """(re, im) views of weights1 in `dtype` (gradients flow back to weights1)."""
        w = self.weights1
        if dtype == torch.float64 and w.dtype != torch.complex128:
            w = w.to(torch.complex128)
        wr = torch.view_as_real(w)
        return wr[..., 0], wr[..., 1]

    def forward(self, x, bias=None, addend=None):
        w_re, w_im = self.weights_re_im(x.dtype)
        return spectral_conv1d(x, w_re, w_im, self.modes1, bias=bias, addend=addend)


def get_grid(x, L):
    """Grid coordinates [B, D] of models/models_1d/utils.py:3-31: a float or int L gives
    linspace(0, L, D) for every row, a tensor L ([B] or [B, 1]) gives L[b] *
    linspace(0, 1, D); anything else raises ValueError."""
    B, D = x.shape[:2]
    if isinstance(L, (float, int)):
        return torch.linspace(0, L, steps=D, dtype=x.dtype, device=x.device).expand(B, D)
    if isinstance(L, torch.Tensor):
        base = torch.linspace(0, 1, steps=D, dtype=x.dtype, device=x.device)
        return L.reshape(B, 1).to(x.dtype) * base
    raise ValueError("L must be a float, int, or a torch.Tensor")


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
    """The reference's FNO corrector (models/models_1d/fno.py:39-105), same constructor
    ``FNO1D(L=16, modes=16, width=64)``, same submodules and parameter names (fc0,
    conv0..conv3 with complex weights1, w0..w3, fc1, fc2), so a state_dict trained with
    the reference loads unchanged; forward(x [B, D], L=None) -> [B, D] with the grid of
    ``get_grid(x, L if L is not None else self.L)``.

    Computed as the reference computes it, with the hidden state kept [B, width, D]
    (contiguous) from the lift to the projection: the Linear layers act on the channel
    axis as channel matmuls (same parameters, same result), each layer's conv_i(x) +
    w_i(x) is one ``inc_spectral_conv1d`` call with w_i's product and bias added in its
    epilogue, and fc1's bias and GELU are one ``inc_bias_gelu`` pass."""

    def __init__(self, L=16, modes=16, width=64):
        super().__init__()
        self.modes1 = modes
        self.width = width
        self.L = L
        self.padding = 2  # unused, as in the reference (its padding lines are commented out)
        self.fc0 = nn.Linear(2, self.width)
        self.conv0 = SpectralConv1d(self.width, self.width, self.modes1)
        self.conv1 = SpectralConv1d(self.width, self.width, self.modes1)
        self.conv2 = SpectralConv1d(self.width, self.width, self.modes1)
        self.conv3 = SpectralConv1d(self.width, self.width, self.modes1)
        self.w0 = nn.Conv1d(self.width, self.width, 1)
        self.w1 = nn.Conv1d(self.width, self.width, 1)
        self.w2 = nn.Conv1d(self.width, self.width, 1)
        self.w3 = nn.Conv1d(self.width, self.width, 1)
        self.fc1 = nn.Linear(self.width, 128)
        self.fc2 = nn.Linear(128, 1)

    def forward(self, x, L=None):
        L = L if L is not None else self.L
        grid = get_grid(x, L)
        h = _channel_linear(self.fc0, torch.stack([x, grid], dim=1))  # [B, width, D]
        layers = ((self.conv0, self.w0), (self.conv1, self.w1), (self.conv2, self.w2), (self.conv3, self.w3))
        for i, (conv, w) in enumerate(layers):
            h = conv(h, bias=w.bias, addend=_channel_mm(w.weight[:, :, 0], h))
            if i + 1 < len(layers):
                h = F.gelu(h)
        h = bias_gelu(_channel_mm(self.fc1.weight, h), self.fc1.bias)
        return _channel_linear(self.fc2, h).squeeze(1)


def fp64_copy(net: nn.Module) -> nn.Module:
    """A float64 copy of a corrector (for FP64 reference runs): real parameters to
    float64 and complex ones (the FNO's weights1) to complex128, which Module.double()
    leaves as complex64."""
    import copy
    out = copy.deepcopy(net).double()
    for m in out.modules():
        for name, prm in list(m.named_parameters(recurse=False)):
            if prm.is_complex() and prm.dtype != torch.complex128:
                setattr(m, name, nn.Parameter(prm.detach().to(torch.complex128)))
    return out
