"""Adaptive-CFL stepping across the GPU (solver_1d.py:148-179), forward and adjoint.

The cooperative kernel spreads a large batch over every SM; the substep sizes come
from the batch-wide max |u| exactly as in the reference.  Forward: against the FP64
oracle's step_adaptive (same substep count, time and state, 1e-5 relative L2).
Gradient: autograd through the reference holds each dt_local constant (it comes
from .item()), so the check is FP64 central differences of the oracle's Euler
substeps with the dt_local sequence of the unperturbed run (1e-4 relative)."""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import burgers as ob
from tests.golden_io import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _case(B, N, eq="viscosity", seed=0, cfl=0.2, dt=0.05):
    rng = np.random.default_rng(seed)
    L = 2 * math.pi
    x = np.arange(N) * (L / N)
    a = rng.uniform(-0.8, 0.8, (B, 4))
    u0 = sum(a[:, k:k + 1] * np.sin((k + 1) * x + 0.7 * k) for k in range(4))
    J = 2
    p = ob.BurgersParams(resolution=N, L=L, dt=dt, nu=rng.uniform(0.005, 0.03, (B, 1)), equation_type=eq,
                         A=rng.uniform(-0.3, 0.3, (B, 1, J)), omega=rng.uniform(-0.5, 0.5, (B, 1, J)),
                         phi=rng.uniform(0, 6.0, (B, 1, J)), l=rng.integers(1, 3, (B, 1, J)).astype(float), x=x,
                         adaptive_CFL=cfl)
    t0 = rng.uniform(0, 1, (B, 1))
    return p, u0, t0


def _solver(p, B, cuda):
    from inc_b200.solvers import BurgersSolverTorch
    f = lambda a: torch.as_tensor(a, dtype=torch.float32, device=cuda)  # noqa: E731
    sp = SimpleNamespace(resolution=p.resolution, dt=p.dt, x=f(p.x), adaptive_CFL=p.adaptive_CFL, L=p.L,
                         nu=f(p.nu), device=cuda, convection_term="WENO", equation_type=p.equation_type,
                         batch_size=B, J=p.A.shape[-1], A=f(p.A), omega=f(p.omega), phi=f(p.phi), l=f(p.l))
    return BurgersSolverTorch(sp)


def _oracle_dts(u, p, t, s):
    """The reference's substep loop (solver_1d.py:148-179): (states, dts, times, final u, count)."""
    target, states, dts, times, sub = float(p.dt), [], [], [], 0
    while target > 0:
        mx = float(np.max(np.abs(u)))
        dtl = min(target, p.adaptive_CFL * p.dx / mx) if mx > 0 else target
        states.append(u)
        dts.append(dtl)
        times.append(t)
        u = u + dtl * ob.rhs(u, p, t, s)
        t = t + dtl
        target -= dtl
        if target > 0 and math.ceil(target / dtl) > 1000:
            break
        sub += 1
    return states, dts, times, u, sub


@pytest.mark.parametrize("B,N,eq", [(4096, 256, "viscosity"), (1000, 128, "learning"), (3, 512, "viscosity"),
                                    (600, 64, "learning")])
def test_adaptive_large_batch_vs_oracle(cuda, B, N, eq):
    p, u0, t0 = _case(B, N, eq, seed=N)
    solver = _solver(p, B, cuda)
    solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
    s0 = 0.05 * np.random.default_rng(1).standard_normal((B, N))
    solver.correction_s = torch.tensor(s0, dtype=torch.float32, device=cuda)
    u = solver.step(torch.tensor(u0, dtype=torch.float32, device=cuda))
    _, dts, _, ref, sub = _oracle_dts(u0, p, t0, s0)
    assert sub >= 3  # several substeps: the grid barrier is exercised
    assert solver.last_substeps == sub
    assert rel_l2(u.cpu().numpy(), ref) < TOL
    np.testing.assert_allclose(solver.t.cpu().numpy(), t0 + sum(dts), rtol=1e-6)


@pytest.mark.parametrize("eq", ["viscosity", "learning"])
def test_adaptive_gradient_vs_fp64_fd(cuda, eq):
    B, N = 5, 64
    p, u0, t0 = _case(B, N, eq, seed=3)
    rng = np.random.default_rng(4)
    s0 = 0.05 * rng.standard_normal((B, N))
    w = rng.standard_normal((B, N))
    solver = _solver(p, B, cuda)
    solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    s = torch.tensor(s0, dtype=torch.float32, device=cuda, requires_grad=True)
    solver.correction_s = s
    out = solver.step(u)
    gu, gs = [g.double().cpu().numpy() for g in torch.autograd.grad(
        (out * torch.tensor(w, dtype=torch.float32, device=cuda)).sum(), (u, s))]
    _, dts, times, _, sub = _oracle_dts(u0, p, t0, s0)
    assert sub >= 3

    def loss(uu, ss):  # the substeps with dt_local held at the unperturbed run's values
        for dtl, t in zip(dts, times):
            uu = uu + dtl * ob.rhs(uu, p, t, ss)
        return float((uu * w).sum())

    h = 1e-6
    for _ in range(3):
        du, dss = rng.standard_normal(u0.shape), rng.standard_normal(s0.shape)
        fdu = (loss(u0 + h * du, s0) - loss(u0 - h * du, s0)) / (2 * h)
        fds = (loss(u0, s0 + h * dss) - loss(u0, s0 - h * dss)) / (2 * h)
        assert abs((gu * du).sum() - fdu) < 1e-4 * max(1.0, abs(fdu))
        assert abs((gs * dss).sum() - fds) < 1e-4 * max(1.0, abs(fds))


def test_adaptive_work_buffer_contract(cuda):
    from inc_b200 import _native as nat
    from inc_b200.adaptive import MAX_SUBSTEPS, run_info
    lib = nat.lib()
    assert lib.inc_burgers_step_adaptive_work_size(0) == -1
    size = lib.inc_burgers_step_adaptive_work_size(MAX_SUBSTEPS)
    assert size >= 64 + 16 * (MAX_SUBSTEPS + 1) and size % 256 == 0
    p, u0, t0 = _case(8, 64, seed=9)
    solver = _solver(p, 8, cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    import ctypes as C
    launch = solver.launch_for(u)  # keeps the tensors its descriptor points to alive
    d = C.byref(launch.desc)
    out = torch.empty_like(u)
    work = torch.empty(size, dtype=torch.uint8, device=cuda)
    subs = torch.zeros(1, dtype=torch.int32, device=cuda)
    s = nat.stream_of(cuda)
    # work is required
    assert lib.inc_burgers_step_adaptive(d, 0.2, MAX_SUBSTEPS, u.data_ptr(), None, None, 0.0, out.data_ptr(),
                                         None, None, subs.data_ptr(), s) == nat.INC_E_INVALID
    rc = lib.inc_burgers_step_adaptive(d, 0.2, MAX_SUBSTEPS, u.data_ptr(), None, None, 0.0, out.data_ptr(),
                                       None, work.data_ptr(), subs.data_ptr(), s)
    assert rc == 0
    executed, err = run_info(work)
    assert err == 0 and executed == int(subs.item()) and executed >= 2
