"""Hybrid rollouts with a corrector network in the loop (GPU).

s = net(u) before every step (trainer_1d.py:168-175), loss = MSE(frames,
target); gradients w.r.t. u0 and every network parameter are compared with
torch autograd through the reference solver in FP64 (golden vectors) and with
FP64 central differences of the oracle."""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import burgers as ob
from tests.golden_io import load, rel_l2

pytestmark = pytest.mark.gpu
HZ = load("hybrid_golden.npz")


@pytest.fixture(autouse=True)
def fp32_corrector():
    """Keep the corrector's convolutions and matmuls in FP32 (cuDNN defaults to TF32)."""
    saved = (torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32)
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    yield
    torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = saved


def _hybrid_burgers(name):
    g = lambda k: HZ[f"{name}.{k}"]  # noqa: E731
    nu = g("nu")
    p = ob.BurgersParams(resolution=int(g("N")), L=float(g("L")), dt=float(g("dt")),
                         nu=(nu if nu.ndim else float(nu)), convection_term=str(g("conv")),
                         equation_type=str(g("eq")))
    return p, g("u0"), str(g("scheme"))


def _net_from_golden(name, net):
    sd = {k: torch.tensor(HZ[f"{name}.param.{k}"]) for k, _ in net.named_parameters()}
    net.load_state_dict(sd, strict=True)
    return net


def _real(a):
    """Complex arrays (the FNO's weights1 and its gradient) as their (re, im) pairs."""
    if isinstance(a, torch.Tensor):
        return (torch.view_as_real(a) if a.is_complex() else a).double().cpu().numpy()
    return np.stack([a.real, a.imag], -1) if np.iscomplexobj(a) else a


def _grads_vs_golden(name, gu, net):
    assert rel_l2(gu.cpu().numpy(), HZ[f"{name}.grad_u"]) < 1e-4
    for k, prm in net.named_parameters():
        assert rel_l2(_real(prm.grad), _real(HZ[f"{name}.pgrad.{k}"])) < 1e-4, k


@pytest.mark.parametrize("name", ["h_burgers_rk3", "h_burgers_euler"])
@pytest.mark.parametrize("ckpt", [None, 2])
def test_burgers_cnn_gradients_vs_reference(cuda, name, ckpt):
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch
    p, u0, scheme = _hybrid_burgers(name)
    B, N = u0.shape
    net = _net_from_golden(name, PeriodicCNN1D(channels=4, kernel=5, layers=4)).to(cuda).float()
    sp = SimpleNamespace(resolution=N, dt=p.dt, x=None, adaptive_CFL=None, L=p.L, nu=p.nu, device=cuda,
                         convection_term="WENO", equation_type="viscosity", batch_size=B,
                         time_scheme="ssprk3" if scheme == "rk3" else "euler")
    solver = BurgersSolverTorch(sp)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    target = torch.tensor(HZ[f"{name}.target"], dtype=torch.float32, device=cuda)
    res, cor = simulate_rollout(net, solver, u, target.shape[1], "INC", checkpoint_every=ckpt)
    loss = torch.mean((res - target) ** 2)
    assert abs(loss.item() - float(HZ[f"{name}.loss"])) < 1e-5 * max(1.0, float(HZ[f"{name}.loss"]))
    net.zero_grad()
    loss.backward()
    _grads_vs_golden(name, u.grad, net)


@pytest.mark.parametrize("ckpt", [None, 2])
def test_ks_fno_gradients_vs_reference(cuda, ckpt):
    from inc_b200.correctors import FNO1D
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import KSSolverTorch
    name = "h_ks"
    N, Ls, dt = int(HZ[f"{name}.N"]), list(HZ[f"{name}.L"]), float(HZ[f"{name}.dt"])
    net = _net_from_golden(name, FNO1D(L=16, modes=4, width=8)).to(cuda).float()  # the reference's FNO1D
    ds = torch.tensor(Ls, dtype=torch.float32, device=cuda)
    solver = KSSolverTorch(SimpleNamespace(resolution=N, dt=dt, device=cuda, domain_size=ds,
                                           alpha=torch.zeros(len(Ls), device=cuda), time_scheme="ETRK2"))
    u = torch.tensor(HZ[f"{name}.u0"], dtype=torch.float32, device=cuda, requires_grad=True)
    target = torch.tensor(HZ[f"{name}.target"], dtype=torch.float32, device=cuda)
    res, _ = simulate_rollout(net, solver, u, target.shape[1], "INC", ds, checkpoint_every=ckpt)
    loss = torch.mean((res - target) ** 2)
    assert abs(loss.item() - float(HZ[f"{name}.loss"])) < 1e-5 * max(1.0, float(HZ[f"{name}.loss"]))
    net.zero_grad()
    loss.backward()
    _grads_vs_golden(name, u.grad, net)


def test_burgers_cnn_fd_check_fp64(cuda):
    """GPU gradients of a CNN-corrected SSP-RK3 rollout vs FP64 central FD (h=1e-6)
    of the oracle with the same network in FP64 on the CPU."""
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch
    torch.manual_seed(0)
    B, N, steps, dt, nu = 3, 64, 4, 0.01, 0.02
    L = 2 * math.pi
    rng = np.random.default_rng(3)
    x = np.arange(N) * (L / N)
    u0 = 0.4 * np.sin(x)[None] + 0.2 * rng.standard_normal((B, 1)) * np.cos(2 * x)[None]
    target = 0.3 * rng.standard_normal((B, steps, N))
    net64 = PeriodicCNN1D(channels=4).double()
    net = PeriodicCNN1D(channels=4).to(cuda)
    net.load_state_dict({k: v.float() for k, v in net64.state_dict().items()})
    sp = SimpleNamespace(resolution=N, dt=dt, x=None, adaptive_CFL=None, L=L, nu=nu, device=cuda,
                         convection_term="WENO", equation_type="viscosity", batch_size=B, time_scheme="ssprk3")
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    res, _ = simulate_rollout(net, BurgersSolverTorch(sp), u, steps, "INC")
    loss = torch.mean((res - torch.tensor(target, dtype=torch.float32, device=cuda)) ** 2)
    loss.backward()
    p = ob.BurgersParams(resolution=N, L=L, dt=dt, nu=nu)

    def L64(uu, net_):
        y, t, acc = uu, 0.0, 0.0
        for k in range(steps):
            with torch.no_grad():
                s = net_(torch.from_numpy(y)).numpy()
            y, t = ob.step_ssprk3(y, p, t, s)
            acc += float(((y - target[:, k]) ** 2).mean()) / steps
        return acc

    h = 1e-6
    du = rng.standard_normal(u0.shape)
    fd = (L64(u0 + h * du, net64) - L64(u0 - h * du, net64)) / (2 * h)
    an = float((u.grad.double().cpu().numpy() * du).sum())
    assert abs(an - fd) < 1e-3 * abs(fd) + 1e-7, (an, fd)
    # along a random direction in parameter space
    dirs = {k: torch.randn_like(v) for k, v in net64.state_dict().items()}

    def shifted(sign):
        m = PeriodicCNN1D(channels=4).double()
        m.load_state_dict({k: v + sign * h * dirs[k] for k, v in net64.state_dict().items()})
        return m

    fdp = (L64(u0, shifted(+1)) - L64(u0, shifted(-1))) / (2 * h)
    anp = sum(float((prm.grad.double().cpu() * dirs[k]).sum()) for k, prm in net.named_parameters())
    assert abs(anp - fdp) < 1e-3 * abs(fdp) + 1e-7, (anp, fdp)
