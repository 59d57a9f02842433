"""The FNO corrector against the reference's own FNO1D (models/models_1d/fno.py:39-105),
whose FP64 outputs and gradients tests/golden/make_golden.py recorded by importing it.

CPU: the same parameters (the reference's state_dict, or the same seed) load into
inc_b200.correctors.FNO1D, whose FP64 copy reproduces the reference to 1e-6: the
reference's Fourier layer writes its mixed modes into a complex64 buffer
(fno.py:33, dtype=torch.cfloat) even in an FP64 run, so its spectral branch
carries FP32 rounding that the FP64 copy here does not.
GPU: the CUDA path (spectral-convolution and bias-GELU kernels, FP32) within 1e-5
(outputs) and 1e-4 (gradients) of the FP64 reference."""
import numpy as np
import pytest
import torch

from tests.golden_io import load, rel_l2

FZ = load("fno_golden.npz")


def _net(case, device="cpu"):
    from inc_b200.correctors import FNO1D
    L, modes, width = (int(v) for v in FZ[f"{case}.kw"])
    torch.manual_seed(int(FZ[f"{case}.seed"]))
    net = FNO1D(L=L, modes=modes, width=width)  # float32 construction: the reference's RNG stream
    if f"{case}.param.fc0.weight" in FZ:
        sd = {}
        for k, p in net.named_parameters():
            a = torch.from_numpy(FZ[f"{case}.param.{k}"])
            sd[k] = torch.view_as_complex(a.contiguous()) if p.is_complex() else a
        net.load_state_dict(sd, strict=True)
    for k, p in net.named_parameters():  # the same parameters as the reference's
        v = torch.view_as_real(p.detach()) if p.is_complex() else p.detach()
        assert abs(float(v.double().sum()) - float(FZ[f"{case}.param_sum.{k}"])) < 1e-6, k
    return net.to(device)


def _real(t):
    return (torch.view_as_real(t) if t.is_complex() else t).double()


def _check(case, net, x, Lt, tol_y, tol_g):
    L0 = int(FZ[f"{case}.kw"][0])
    with torch.no_grad():
        assert rel_l2(net(x).cpu().numpy(), FZ[f"{case}.y_none"]) < tol_y      # L=None -> self.L
        assert rel_l2(net(x, 5.0).cpu().numpy(), FZ[f"{case}.y_float"]) < tol_y  # a float L
        assert net.L == L0
    xg = x.clone().requires_grad_(True)
    y = net(xg, Lt)                                                              # a per-row tensor L
    assert rel_l2(y.detach().cpu().numpy(), FZ[f"{case}.y_tensor"]) < tol_y
    w = torch.from_numpy(FZ[f"{case}.w"]).to(x)
    grads = torch.autograd.grad((y * w).sum(), [xg] + list(net.parameters()))
    assert rel_l2(grads[0].cpu().numpy(), FZ[f"{case}.grad_x"]) < tol_g
    g = torch.Generator().manual_seed(int(FZ[f"{case}.seed"]))
    for (k, p), gp in zip(net.named_parameters(), grads[1:]):
        d = torch.randn(p.shape, generator=g, dtype=torch.float64)
        if p.is_complex():
            d = torch.stack([d, torch.randn(p.shape, generator=g, dtype=torch.float64)], -1)
        proj = float((_real(gp).cpu() * d).sum())
        ref = float(FZ[f"{case}.pgrad_proj.{k}"])
        assert abs(proj - ref) <= tol_g * max(abs(ref), 1e-3 * float(np.abs(FZ[f"{case}.grad_x"]).max())), k
        if f"{case}.pgrad.{k}" in FZ:
            assert rel_l2(_real(gp).cpu().numpy(), FZ[f"{case}.pgrad.{k}"]) < tol_g, k


@pytest.mark.parametrize("case", ["f_small", "f_bench"])
def test_fno_fp64_matches_reference(case):
    from inc_b200.correctors import fp64_copy
    net = fp64_copy(_net(case))
    x = torch.from_numpy(FZ[f"{case}.x"])
    _check(case, net, x, torch.from_numpy(FZ[f"{case}.Lt"]), 1e-6, 1e-5)


def test_fno_state_dict_names_are_the_reference_ones():
    net = _net("f_small")
    names = [k for k, _ in net.named_parameters()]
    assert names[:2] == ["fc0.weight", "fc0.bias"] and "conv3.weights1" in names and names[-1] == "fc2.bias"
    assert net.conv0.weights1.dtype == torch.complex64 and net.conv0.modes1 == 4
    from inc_b200.correctors import get_grid
    with pytest.raises(ValueError):
        get_grid(torch.zeros(2, 8), "16")


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["f_small", "f_bench"])
def test_fno_cuda_matches_reference(cuda, case):
    saved = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        net = _net(case, cuda)
        x = torch.from_numpy(FZ[f"{case}.x"]).float().to(cuda)
        Lt = torch.from_numpy(FZ[f"{case}.Lt"]).float().to(cuda)
        _check(case, net, x, Lt, 1e-5, 1e-4)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = saved
