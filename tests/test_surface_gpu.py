"""The rest of the reference solvers' public surface on the drop-in classes (GPU):
Burgers calc_nonlinear_weno / _FDM, calc_linear, _compute_source,
_apply_corrections, D2_T / D1_T; KS calc_linear, calc_nonlinear, etrk2_step,
etd1_step (solver_1d.py:87-146, :225-278).  Against the reference's golden
vectors (FP64) and the FP64 oracle; tolerance 1e-5 relative L2 (FP32 state)."""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import burgers as ob
from oracle import ks as oks
from tests.golden_io import burgers_case, ks_case, load, rel_l2

pytestmark = pytest.mark.gpu
BZ = load("burgers_golden.npz")
KZ = load("ks_golden.npz")
TOL = 1e-5


def _burgers(N, conv="WENO", eq="viscosity", nu=0.01, B=3, **kw):
    from inc_b200.solvers import BurgersSolverTorch
    sp = SimpleNamespace(resolution=N, dt=0.01, x=kw.pop("x", None), adaptive_CFL=None, L=2 * math.pi, nu=nu,
                         device="cuda", convection_term=conv, equation_type=eq, batch_size=B, **kw)
    return BurgersSolverTorch(sp)


def test_burgers_terms_vs_reference_golden(cuda):
    u = torch.tensor(BZ["op_u"], dtype=torch.float32, device=cuda)  # 3 x 32, nu = 0.01 (make_golden.py)
    s = _burgers(32)
    assert rel_l2(s.calc_nonlinear_weno(u).cpu().numpy(), BZ["op_nonlinear_weno"]) < TOL
    assert rel_l2(s.calc_nonlinear(u).cpu().numpy(), BZ["op_nonlinear_weno"]) < TOL
    assert rel_l2(s.calc_linear(u).cpu().numpy(), BZ["op_linear"]) < TOL
    d2 = s.D2_T.T.cpu().double().numpy()
    assert np.allclose(u.cpu().double().numpy() @ d2.T * 0.01, BZ["op_linear"], rtol=1e-4, atol=1e-4)
    with pytest.raises(AttributeError):
        s.D1_T  # noqa: B018  WENO convection: the reference defines no D1_T


@pytest.mark.parametrize("name", ["euler_learning", "euler_linear_fdm", "rk3_linear"])
def test_burgers_terms_vs_oracle(cuda, name):
    from inc_b200.solvers import BurgersSolverTorch
    from tests.test_burgers_gpu import _sim_params
    p, u0, t0, s0, _ = burgers_case(BZ, name)
    B = u0.shape[0]
    solver = BurgersSolverTorch(_sim_params(p, B))
    solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    nl = ob.nonlinear_weno(u0, p.dx) if p.convection_term == "WENO" else ob.nonlinear_fdm(u0, p.dx)
    got = solver.calc_nonlinear(u).cpu().numpy()
    assert rel_l2(got, nl) < TOL
    assert rel_l2(solver.calc_linear(u).cpu().numpy(), ob.linear(u0, p.nu, p.dx)) < TOL
    src = solver._compute_source(u)
    ref_src = ob.source(u0, p, t0)
    assert rel_l2(src.cpu().numpy(), ref_src) < TOL
    if p.convection_term == "FDM":
        d1 = solver.D1_T.T.cpu().double().numpy()
        assert np.allclose(-u0 * (u0 @ d1.T), nl, rtol=1e-4, atol=1e-4)
    solver.correction_s = torch.ones_like(u)
    assert torch.equal(solver._apply_corrections(src), src + 1.0)
    # a step is u + dt (nonlinear + linear + source + s) (solver_1d.py:186-192)
    if name.startswith("euler"):
        solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
        solver.correction_s = None
        rhs = solver.calc_nonlinear(u) + solver.calc_linear(u) + src
        stepped = solver.step(u)
        assert rel_l2(stepped.cpu().numpy(), (u + p.dt * rhs).cpu().numpy()) < 1e-6


def test_burgers_terms_refuse_autograd(cuda):
    s = _burgers(32)
    u = torch.zeros(3, 32, device=cuda, requires_grad=True)
    with pytest.raises(RuntimeError):
        s.calc_linear(u)
    viscous = _burgers(32)
    assert viscous._compute_source(u.detach()) == 0.0


def _ks(N, dt, scheme, Ls):
    from inc_b200.solvers import KSSolverTorch
    ds = torch.tensor(Ls, dtype=torch.float32, device="cuda")
    return KSSolverTorch(SimpleNamespace(resolution=N, dt=dt, device="cuda", domain_size=ds,
                                         alpha=torch.zeros_like(ds), time_scheme=scheme)), ds


@pytest.mark.parametrize("name", [str(n) for n in KZ["cases"]])
def test_ks_substep_vs_reference_golden(cuda, name):
    c = ks_case(KZ, name)
    solver, ds = _ks(c["N"], c["dt"], c["scheme"], list(c["L"]))
    f = lambda a: None if a is None else torch.tensor(a, dtype=torch.float32, device=cuda)  # noqa: E731
    solver.correction_s, solver.correction_u = f(c["s"]), f(c["cu"])  # correction_u: not used by a substep
    sub = solver.etrk2_step if c["scheme"] == "ETRK2" else solver.etd1_step
    got = sub(f(c["u0"]), ds).cpu().numpy()
    assert rel_l2(got, KZ[f"{name}.substep"]) < TOL


@pytest.mark.parametrize("scheme", ["ETRK2", "ETD1"])
def test_ks_substep_gradient_vs_fp64_fd(cuda, scheme):
    N, dt = 64, (0.2 if scheme == "ETRK2" else 0.05)
    Ls = [40.0, 40.0, 52.0]
    solver, ds = _ks(N, dt, scheme, Ls)
    rng = np.random.default_rng(3)
    from tests.test_ks_gpu import _u0
    u0 = _u0(3, N, Ls, 12)
    s0 = 0.01 * rng.standard_normal((3, N))
    w = rng.standard_normal((3, N))
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    s = torch.tensor(s0, dtype=torch.float32, device=cuda, requires_grad=True)
    solver.correction_s = s
    sub = solver.etrk2_step if scheme == "ETRK2" else solver.etd1_step
    out = sub(u, ds)
    ref = (oks.etrk2_step if scheme == "ETRK2" else oks.etd1_step)(u0, Ls, dt, s0)
    assert rel_l2(out.detach().cpu().numpy(), ref) < TOL
    gu, gs = [g.double().cpu().numpy() for g in torch.autograd.grad((out * torch.tensor(
        w, dtype=torch.float32, device=cuda)).sum(), (u, s))]
    fn = oks.etrk2_step if scheme == "ETRK2" else oks.etd1_step
    h = 1e-6
    for _ in range(3):
        du, dss = rng.standard_normal(u0.shape), rng.standard_normal(s0.shape)
        fdu = float(((fn(u0 + h * du, Ls, dt, s0) - fn(u0 - h * du, Ls, dt, s0)) * w).sum()) / (2 * h)
        fds = float(((fn(u0, Ls, dt, s0 + h * dss) - fn(u0, Ls, dt, s0 - h * dss)) * w).sum()) / (2 * h)
        assert abs((gu * du).sum() - fdu) < 1e-4 * max(1.0, abs(fdu))
        assert abs((gs * dss).sum() - fds) < 1e-4 * max(1.0, abs(fds))


@pytest.mark.parametrize("N", [16, 64, 256, 512])
def test_ks_calc_linear_and_nonlinear(cuda, N):
    B = 5  # odd: a lone row in the row-pair FFT
    Ls = [30.0 + 11 * i for i in range(B)]
    solver, ds = _ks(N, 0.1, "ETRK2", Ls)
    lop, wn = solver.calc_linear(ds)
    rlop, rwn = oks.linear_operator(Ls, N)
    assert rel_l2(lop.cpu().numpy(), rlop) < TOL and rel_l2(wn.cpu().numpy(), rwn) < TOL
    from tests.test_ks_gpu import _u0
    u0 = _u0(B, N, Ls, N)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    nl = solver.calc_nonlinear(u, wn)
    assert rel_l2(nl.detach().cpu().numpy(), oks.nonlinear(u0, rwn)) < TOL
    # gradient of a real function of the complex output, against torch's FFT on the same inputs
    w = torch.randn(B, N, dtype=torch.complex64, device=cuda)
    g, = torch.autograd.grad((nl * w).real.sum(), (u,))
    u2 = u.detach().double().requires_grad_(True)
    nl2 = -0.5 * wn.to(torch.complex128) * torch.fft.fft(u2 * u2)
    g2, = torch.autograd.grad((nl2 * w.to(torch.complex128)).real.sum(), (u2,))
    assert rel_l2(g.cpu().numpy(), g2.cpu().numpy()) < TOL
