"""FNO spectral convolution on the GPU (inc_spectral_conv1d and its adjoint).

SpectralConv1d.forward (models/models_1d/fno.py:26-37) is rfft, the lowest
`modes` modes times complex [cin][cout][modes] weights, irfft.  The kernel and
its hand-written adjoint are checked against torch's FFT formulation of the
same layer evaluated in FP64 (forward, autograd's input and weight gradients),
over every supported row length, edge widths and mode counts, batches of one
and odd batches, non-contiguous inputs, and shapes that take the torch path."""
import pytest
import torch

from inc_b200 import _native as nat
from inc_b200.correctors import (FNO1D, SPECTRAL_CONV_N, SpectralConv1d, bias_gelu, spectral_conv1d,
                                 spectral_conv1d_torch, spectral_conv_supported)

pytestmark = pytest.mark.gpu
TOL = 1e-5  # max abs error over max abs FP64 value


def _case(B, W, n, modes, seed=0):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(B, W, n, generator=g, dtype=torch.float64)
    scale = 1.0 / (W * W)
    w_re = scale * torch.rand(W, W, modes, generator=g, dtype=torch.float64)
    w_im = scale * torch.rand(W, W, modes, generator=g, dtype=torch.float64)
    gy = torch.randn(B, W, n, generator=g, dtype=torch.float64)
    return x, w_re, w_im, gy


def _rel(a, ref):
    return (a.detach().double().cpu() - ref).abs().max().item() / max(ref.abs().max().item(), 1e-30)


def _check(B, W, n, modes, seed=0):
    x, w_re, w_im, gy = _case(B, W, n, modes, seed)
    # FP64 reference with autograd
    xr, wr, wi = (t.clone().requires_grad_(True) for t in (x, w_re, w_im))
    yr = spectral_conv1d_torch(xr, wr, wi, modes)
    yr.backward(gy)
    # the kernel
    xc, wrc, wic = (t.float().cuda().requires_grad_(True) for t in (x, w_re, w_im))
    assert spectral_conv_supported(xc, wrc, wic, min(modes, n // 2 + 1))
    y = spectral_conv1d(xc, wrc, wic, modes)
    y.backward(gy.float().cuda())
    errs = dict(y=_rel(y, yr.detach()), gx=_rel(xc.grad, xr.grad), gw_re=_rel(wrc.grad, wr.grad),
                gw_im=_rel(wic.grad, wi.grad))
    assert all(e < TOL for e in errs.values()), (B, W, n, modes, errs)
    return errs


_LANES = {16: 4, 32: 8, 64: 16, 128: 32, 256: 32, 512: 32}  # lanes per row pair of each n's transform
_N_MODES = sorted({(n, m) for n in SPECTRAL_CONV_N for m in (1, _LANES[n], min(16, n // 2), min(32, n // 2))})


@pytest.mark.parametrize("n,modes", _N_MODES)
def test_every_row_length_and_split_path(n, modes):
    # modes <= lanes: the two rows' coefficients split by one exchange; above: the full mirror split
    _check(3, 8, n, modes, seed=n + modes)


@pytest.mark.parametrize("W,modes", [(2, 1), (6, 5), (64, 16), (128, 32), (64, 32)])
def test_widths_and_modes(W, modes):
    _check(5, W, 256, modes, seed=W + modes)


def test_fno_benchmark_shape_and_max_modes():
    _check(17, 64, 256, 16, seed=3)   # the KS FNO configuration (width 64, 16 modes)
    _check(2, 16, 16, 8, seed=4)      # modes = n/2: the highest mode the kernel takes
    _check(1, 4, 512, 32, seed=5)     # one trajectory, the longest rows


def test_non_contiguous_input_and_unused_weight_modes():
    # x arrives permuted from the lifting layer; the layer holds more weight modes than n/2
    x, w_re, w_im, gy = _case(4, 8, 32, 20, seed=6)
    xp = x.permute(0, 2, 1).contiguous().permute(0, 2, 1)
    xr, wr, wi = (t.clone().requires_grad_(True) for t in (xp, w_re, w_im))
    yr = spectral_conv1d_torch(xr, wr, wi, 16)
    yr.backward(gy)
    xc = x.float().cuda().permute(0, 2, 1).contiguous().permute(0, 2, 1).requires_grad_(True)
    assert not xc.is_contiguous()
    wrc, wic = (t.float().cuda().requires_grad_(True) for t in (w_re, w_im))
    y = spectral_conv1d(xc, wrc, wic, 16)
    y.backward(gy.float().cuda())
    assert _rel(y, yr.detach()) < TOL and _rel(xc.grad, xr.grad) < TOL
    assert _rel(wrc.grad, wr.grad) < TOL and _rel(wic.grad, wi.grad) < TOL
    assert wrc.grad[..., 16:].abs().max().item() == 0.0


def test_shapes_outside_the_kernel_take_the_torch_path():
    # odd width, modes reaching the Nyquist bin, and a non-power-of-two length
    for (B, W, n, modes) in [(2, 5, 64, 8), (2, 8, 16, 9), (2, 8, 48, 8)]:
        x, w_re, w_im, _ = _case(B, W, n, modes)
        xc, wrc, wic = (t.float().cuda() for t in (x, w_re, w_im))
        assert not spectral_conv_supported(xc, wrc, wic, min(modes, n // 2 + 1))
        y = spectral_conv1d(xc, wrc, wic, modes)
        assert _rel(y, spectral_conv1d_torch(x, w_re, w_im, modes)) < TOL


def test_c_abi_rejects_unsupported_shapes():
    lib = nat.lib()
    x = torch.zeros(2, 6, 64, device="cuda")
    y = torch.empty_like(x)
    w = torch.zeros(6, 6, 8, device="cuda")
    s = nat.stream_of(x.device)
    modes = torch.empty(2, 6, 8, 2, device="cuda")
    work = torch.empty(2 * 8 * 6 * (2 + 6), device="cuda")
    fwd = (x.data_ptr(), w.data_ptr(), w.data_ptr(), None, None, y.data_ptr(), modes.data_ptr(), work.data_ptr())
    bwd = (x.data_ptr(), w.data_ptr(), w.data_ptr(), y.data_ptr(), modes.data_ptr(), work.data_ptr())
    assert lib.inc_spectral_conv1d(*fwd, 2, 5, 64, 8, s) != 0      # odd width
    assert lib.inc_spectral_conv1d(*fwd, 2, 6, 64, 33, s) != 0     # modes > 32
    assert lib.inc_spectral_conv1d(*fwd, 2, 6, 48, 8, s) != 0      # n not a power of two
    assert lib.inc_spectral_conv1d_bwd(*bwd, 2, 6, 64, 0, s) != 0  # no modes
    assert "spectral_conv" in nat.last_error()
    assert lib.inc_spectral_conv1d(*fwd[:6], None, None, 2, 6, 64, 8, s) != 0  # no mode buffers
    assert lib.inc_spectral_conv1d(*fwd, 2, 6, 64, 8, s) == 0
    torch.cuda.synchronize()


@pytest.mark.parametrize("n,W", [(512, 64), (64, 6)])
def test_layer_sum_with_bias_and_addend(n, W):
    """spectral(x) + bias[:, None] + addend in one kernel: values and the gradients
    of x, the weights, the bias (from the backward's DC coefficient) and the addend."""
    x, w_re, w_im, gy = _case(3, W, n, 16 if n > 64 else 8, seed=n)
    modes = w_re.shape[-1]
    g = torch.Generator().manual_seed(7)
    bias = torch.randn(W, generator=g, dtype=torch.float64)
    add = torch.randn(3, W, n, generator=g, dtype=torch.float64)
    ref_in = [t.clone().requires_grad_(True) for t in (x, w_re, w_im, bias, add)]
    yr = spectral_conv1d_torch(*ref_in[:3], modes) + ref_in[3][:, None] + ref_in[4]
    yr.backward(gy)
    cu_in = [t.float().cuda().requires_grad_(True) for t in (x, w_re, w_im, bias, add)]
    y = spectral_conv1d(*cu_in[:3], modes, bias=cu_in[3], addend=cu_in[4])
    assert y.grad_fn is not None and "SpectralConv1dFn" in type(y.grad_fn).__name__
    y.backward(gy.float().cuda())
    assert _rel(y, yr.detach()) < TOL
    for a, r in zip(cu_in, ref_in):
        assert _rel(a.grad, r.grad) < TOL


def test_fno_corrector_matches_fp64():
    from inc_b200.correctors import fp64_copy
    torch.manual_seed(0)
    net = FNO1D(L=16, modes=16, width=64)
    u = torch.randn(6, 256, dtype=torch.float64)
    L = torch.full((6,), 64.0, dtype=torch.float64)
    ref_net = fp64_copy(net)
    ur = u.clone().requires_grad_(True)
    sr = ref_net(ur, L)
    gs = torch.randn_like(sr)
    sr.backward(gs)
    saved = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        net = net.cuda()
        uc = u.float().cuda().requires_grad_(True)
        s = net(uc, L.float().cuda())
        s.backward(gs.float().cuda())
    finally:
        torch.backends.cuda.matmul.allow_tf32 = saved
    assert _rel(s, sr.detach()) < 1e-5
    assert _rel(uc.grad, ur.grad) < 1e-4
    for (name, p), (_, pr) in zip(net.named_parameters(), ref_net.named_parameters()):
        g, gr = p.grad, pr.grad
        if g.is_complex():
            g, gr = torch.view_as_real(g), torch.view_as_real(gr)
        assert _rel(g, gr) < 1e-4, name
    assert isinstance(net.conv0, SpectralConv1d)


@pytest.mark.parametrize("B,C,n", [(3, 128, 512), (2, 8, 16), (1, 5, 36)])
def test_bias_gelu_matches_fp64(B, C, n):
    """The FNO projection's gelu(h + b) (inc_bias_gelu and its backward) against torch in FP64."""
    g = torch.Generator().manual_seed(B * C + n)
    h = 3 * torch.randn(B, C, n, generator=g, dtype=torch.float64)
    b = torch.randn(C, generator=g, dtype=torch.float64)
    gy = torch.randn(B, C, n, generator=g, dtype=torch.float64)
    hr, br = h.clone().requires_grad_(True), b.clone().requires_grad_(True)
    yr = torch.nn.functional.gelu(hr + br[:, None])
    yr.backward(gy)
    hc, bc = h.float().cuda().requires_grad_(True), b.float().cuda().requires_grad_(True)
    y = bias_gelu(hc, bc)
    assert "BiasGeluFn" in type(y.grad_fn).__name__
    y.backward(gy.float().cuda())
    assert _rel(y, yr.detach()) < TOL
    assert _rel(hc.grad, hr.grad) < TOL
    assert _rel(bc.grad, br.grad) < TOL


def test_bias_gelu_c_abi_rejects_bad_shapes():
    lib = nat.lib()
    h = torch.zeros(2, 4, 18, device="cuda")
    b = torch.zeros(4, device="cuda")
    s = nat.stream_of(h.device)
    assert lib.inc_bias_gelu(h.data_ptr(), b.data_ptr(), h.data_ptr(), 8, 18, 4, s) != 0   # n not a multiple of 4
    assert lib.inc_bias_gelu(h.data_ptr(), b.data_ptr(), h.data_ptr(), 8, 16, 3, s) != 0   # rows % channels
    assert "bias_gelu" in nat.last_error()
