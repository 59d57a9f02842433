"""Burgers CUDA path vs the FP64 oracle and the reference's golden vectors (GPU)."""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import burgers as ob
from tests.golden_io import burgers_case, load, rel_l2

pytestmark = pytest.mark.gpu
BZ = load("burgers_golden.npz")
TOL = 1e-5  # relative L2 vs FP64 (FP32 state throughout)


def _sim_params(p: ob.BurgersParams, B, scheme="euler", cpt=0, device="cuda"):
    f = lambda a: None if a is None else torch.as_tensor(a, dtype=torch.float32, device=device)  # noqa: E731
    nu = f(p.nu) if isinstance(p.nu, np.ndarray) else p.nu
    return SimpleNamespace(resolution=p.resolution, dt=p.dt, x=f(p.x) if p.x is not None else None,
                           adaptive_CFL=p.adaptive_CFL, L=p.L, nu=nu, device=device,
                           convection_term=p.convection_term, equation_type=p.equation_type, batch_size=B,
                           beta=f(p.beta) if isinstance(p.beta, np.ndarray) else p.beta,
                           J=(p.A.shape[-1] if p.A is not None else 0), A=f(p.A), omega=f(p.omega), phi=f(p.phi),
                           l=f(p.l), time_scheme=scheme, cells_per_thread=cpt)


def _rand_u0(B, N, seed, L=2 * math.pi):
    rng = np.random.default_rng(seed)
    x = np.arange(N) * (L / N)
    a = rng.uniform(-0.5, 0.5, (B, 5))
    ph = rng.uniform(0, 2 * np.pi, (B, 5))
    k = np.arange(1, 6)
    return (a[:, :, None] * np.sin(k[None, :, None] * x[None, None, :] + ph[:, :, None])).sum(1)


@pytest.mark.parametrize("name", [str(n) for n in BZ["cases"] if not str(n).startswith("adaptive")])
def test_golden_rollouts(cuda, name):
    from inc_b200.solvers import BurgersSolverTorch
    p, u0, t0, s, scheme = burgers_case(BZ, name)
    frames = BZ[f"{name}.frames"]
    B = u0.shape[0]
    solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3" if scheme == "rk3" else "euler"))
    solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
    solver.correction_s = None if s is None else torch.tensor(s, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    for k in range(frames.shape[1]):
        u = solver.step(u)
        assert rel_l2(u.cpu().numpy(), frames[:, k]) < TOL, (name, k)


def test_golden_adaptive(cuda):
    from inc_b200.solvers import BurgersSolverTorch
    name = "adaptive_visc"
    p, u0, t0, s, _ = burgers_case(BZ, name)
    frames = BZ[f"{name}.frames"]
    solver = BurgersSolverTorch(_sim_params(p, u0.shape[0]))
    solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    for k in range(frames.shape[1]):
        u = solver.step(u)
        assert rel_l2(u.cpu().numpy(), frames[:, k]) < TOL, k
    assert solver.last_substeps == int(BZ[f"{name}.substeps"])


def test_weno_reconstruction(cuda):
    from inc_b200.ops import weno_reconstruction
    rng = np.random.default_rng(5)
    for n in (8, 16, 32, 64, 128, 256, 512):
        f = rng.standard_normal((7, n))
        for d in ("left", "right"):
            got = weno_reconstruction(torch.tensor(f, dtype=torch.float32, device=cuda), d).cpu().numpy()
            assert rel_l2(got, ob.weno_reconstruction(f, d)) < 2e-6, (n, d)
    with pytest.raises(ValueError):
        weno_reconstruction(torch.zeros(2, 16, device=cuda), "up")


@pytest.mark.parametrize("n,cpt", [(8, 4), (16, 4), (32, 4), (32, 8), (64, 4), (64, 8), (128, 4), (128, 8),
                                   (128, 16), (256, 8), (256, 16), (512, 16),
                                   (64, 1), (128, 1), (128, 2), (256, 1), (256, 2), (512, 1)])
@pytest.mark.parametrize("scheme", ["euler", "ssprk3"])
def test_shapes_vs_oracle(cuda, n, cpt, scheme):
    from inc_b200.solvers import BurgersSolverTorch
    B = 5  # odd: partial row groups
    L = 2 * math.pi
    dt = 0.2 * (L / n)
    p = ob.BurgersParams(resolution=n, L=L, dt=dt, nu=0.01)
    u0 = _rand_u0(B, n, n)
    solver = BurgersSolverTorch(_sim_params(p, B, scheme, cpt))
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    ref, t = u0, 0.0
    fn = ob.step_ssprk3 if scheme == "ssprk3" else ob.step_euler
    for _ in range(10):
        u = solver.step(u)
        ref, t = fn(ref, p, t)
    assert rel_l2(u.cpu().numpy(), ref) < TOL


def test_config0_ssprk3_200_steps(cuda):
    """Plain Burgers: N=128, nu=0.01, dt=0.01, 200 SSP-RK3 steps, batch 32, s=0."""
    from inc_b200.solvers import BurgersSolverTorch
    from inc_b200.workloads import burgers_plain_config
    cfg = burgers_plain_config()
    p = ob.BurgersParams(resolution=cfg["N"], L=cfg["L"], dt=cfg["dt"], nu=cfg["nu"])
    solver = BurgersSolverTorch(_sim_params(p, cfg["B"], "ssprk3"))
    u = torch.tensor(cfg["u0"], dtype=torch.float32, device=cuda)
    ref, t = cfg["u0"], 0.0
    frames, rframes = [], []
    for _ in range(cfg["steps"]):
        u = solver.step(u)
        ref, t = ob.step_ssprk3(ref, p, t)
        frames.append(u)
        rframes.append(ref)
    got = torch.stack(frames, 1).cpu().numpy()
    assert rel_l2(got, np.stack(rframes, 1)) < TOL


def test_fused_rollout_matches_steps(cuda):
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    n, B = 128, 9
    p = ob.BurgersParams(resolution=n, L=2 * math.pi, dt=0.01, nu=0.02)
    u0 = torch.tensor(_rand_u0(B, n, 1), dtype=torch.float32, device=cuda)
    s = 0.1 * torch.randn(B, n, device=cuda)
    for scheme in ("euler", "ssprk3"):
        a = BurgersSolverTorch(_sim_params(p, B, scheme))
        a.correction_s = s
        u, frames = u0, []
        for _ in range(23):
            u = a.step(u)
            frames.append(u)
        b = BurgersSolverTorch(_sim_params(p, B, scheme))
        fused = burgers_rollout(b, u0, 23, s=s)
        # the fused launch carries the rounding error of each update into the next step
        # (compensated summation), the per-step launches cannot: equal up to that rounding
        stepped = torch.stack(frames, 1)
        assert rel_l2(fused.cpu().numpy(), stepped.cpu().numpy()) < 1e-6, scheme
        fn = ob.step_ssprk3 if scheme == "ssprk3" else ob.step_euler
        ref, t, rf = u0.cpu().double().numpy(), 0.0, []
        for _ in range(23):
            ref, t = fn(ref, p, t, s.cpu().double().numpy())
            rf.append(ref)
        rf = np.stack(rf, 1)
        assert rel_l2(fused.cpu().numpy(), rf) <= rel_l2(stepped.cpu().numpy(), rf) * 1.5 + 1e-9, scheme


def test_simulate_rollout_dropin_no_model(cuda):
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch
    n, B = 64, 4
    p = ob.BurgersParams(resolution=n, L=2 * math.pi, dt=0.01, nu=0.01)
    u0 = _rand_u0(B, n, 3)
    solver = BurgersSolverTorch(_sim_params(p, B))
    res, cor = simulate_rollout(None, solver, torch.tensor(u0, dtype=torch.float32, device=cuda), 12, None)
    assert cor is None and res.shape == (B, 12, n)
    assert rel_l2(res.cpu().numpy(), ob.rollout(u0, p, 12)) < TOL


@pytest.mark.parametrize("name", [str(n) for n in BZ["grad_cases"]])
def test_step_gradients_vs_reference_autograd(cuda, name):
    """Hand-written adjoint vs torch autograd through the (fixed) reference, FP64."""
    from inc_b200.solvers import BurgersSolverTorch
    p, u0, t0, s, scheme = burgers_case(BZ, name)
    w = torch.tensor(BZ[f"{name}.w"], dtype=torch.float32, device=cuda)
    B = u0.shape[0]
    solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3" if scheme == "rk3" else "euler"))
    solver.t = torch.tensor(t0, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    st = torch.tensor(s, dtype=torch.float32, device=cuda, requires_grad=True)
    solver.correction_s = st
    x, loss = u, 0.0
    for k in range(w.shape[1]):
        x = solver.step(x)
        loss = loss + (x * w[:, k]).sum()
    gu, gs = torch.autograd.grad(loss, (u, st))
    assert rel_l2(gu.cpu().numpy(), BZ[f"{name}.grad_u"]) < 1e-4
    assert rel_l2(gs.cpu().numpy(), BZ[f"{name}.grad_s"]) < 1e-4


@pytest.mark.parametrize("scheme", ["euler", "ssprk3"])
def test_rollout_backward_matches_stepwise(cuda, scheme):
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    n, B, steps = 256, 6, 19
    p = ob.BurgersParams(resolution=n, L=2 * math.pi, dt=0.004, nu=0.01)
    u0 = torch.tensor(_rand_u0(B, n, 8), dtype=torch.float32, device=cuda)
    s0 = 0.05 * torch.randn(B, n, device=cuda)
    w = torch.randn(B, steps, n, device=cuda)
    # step by step (per-step adjoint kernels)
    a = BurgersSolverTorch(_sim_params(p, B, scheme))
    u = u0.clone().requires_grad_(True)
    s = s0.clone().requires_grad_(True)
    a.correction_s = s
    x, frames = u, []
    for _ in range(steps):
        x = a.step(x)
        frames.append(x)
    ga = torch.autograd.grad((torch.stack(frames, 1) * w).sum(), (u, s))
    # fused rollout with checkpoint every 8
    b = BurgersSolverTorch(_sim_params(p, B, scheme))
    u2 = u0.clone().requires_grad_(True)
    s2 = s0.clone().requires_grad_(True)
    fr = burgers_rollout(b, u2, steps, s=s2, ckpt_every=8)
    gb = torch.autograd.grad((fr * w).sum(), (u2, s2))
    # the fused forward carries its update rounding from step to step (compensated
    # summation) and the per-step launches do not, so the states the two backward
    # passes linearise at differ by FP32 rounding: equal to 1e-5, not to the last bit
    for x1, x2 in zip(ga, gb):
        assert rel_l2(x2.cpu().numpy(), x1.cpu().numpy()) < 1e-5


_WARP_CPT = {64: 4, 128: 4, 256: 8, 512: 16}


@pytest.mark.parametrize("n", [64, 128, 256, 512])
@pytest.mark.parametrize("scheme", ["euler", "ssprk3"])
@pytest.mark.parametrize("conv,eq", [("WENO", "viscosity"), ("WENO", "linear"), ("FDM", "learning")])
def test_wide_adjoint_matches_warp_adjoint(cuda, n, scheme, conv, eq):
    """The one-cell-per-thread adjoint (small batches) against the warp-layout
    adjoint: a step's VJP and a checkpointed rollout's gradient w.r.t. u0 and
    s, with per-row nu, the linear or forcing source and per-row time."""
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    B, L, J = 5, 2 * math.pi, 2
    g = torch.Generator().manual_seed(n + len(eq))
    rnd = lambda *shape: torch.rand(*shape, generator=g).to(cuda)  # noqa: E731
    u0 = torch.tensor(_rand_u0(B, n, n), dtype=torch.float32, device=cuda)
    s0 = 0.05 * (rnd(B, n) - 0.5)
    t0 = rnd(B, 1)

    def solver(cpt):
        sp = SimpleNamespace(resolution=n, dt=0.2 / n, x=torch.arange(n, device=cuda) * (L / n),
                             adaptive_CFL=None, L=L, nu=0.005 + 0.02 * rnd(B, 1), device=cuda,
                             convection_term=conv, equation_type=eq, batch_size=B, beta=rnd(B, 1) - 0.5, J=J,
                             A=0.3 * rnd(B, J), omega=rnd(B, J), phi=6 * rnd(B, J),
                             l=torch.randint(1, 4, (B, J), generator=g).float().to(cuda),
                             time_scheme=scheme, cells_per_thread=cpt)
        return sp

    g_state = g.get_state()
    out = []
    for cpt in (1, _WARP_CPT[n]):
        g.set_state(g_state)  # the same random parameters for both layouts
        slv = BurgersSolverTorch(solver(cpt))
        slv.t = t0.clone()
        u = u0.clone().requires_grad_(True)
        s = s0.clone().requires_grad_(True)
        slv.correction_s = s
        w = torch.sin(torch.arange(n, device=cuda) * 0.3)
        step_g = torch.autograd.grad((slv.step(u) * w).sum(), (u, s))
        slv.t = t0.clone()
        fr = burgers_rollout(slv, u, 11, s=s, ckpt_every=4)
        wf = torch.cos(torch.arange(11 * n, device=cuda).reshape(11, n) * 0.01)
        roll_g = torch.autograd.grad((fr * wf).sum(), (u, s))
        out.append(step_g + roll_g)
    for a, b in zip(*out):
        assert torch.isfinite(a).all()
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 2e-5


@pytest.mark.parametrize("n,B", [(128, 40), (128, 60), (128, 100), (256, 40), (256, 100), (64, 49)])
def test_wide_adjoint_forms_by_batch(cuda, n, B):
    """The one-cell-per-thread adjoint takes one of three forms by batch size (three
    CTAs per row up to 49 rows at n <= 128, two CTAs per row up to 74, two thread
    groups on one CTA above); each against the warp-layout adjoint of the same
    checkpointed rollout (three segments), gradients w.r.t. u0 and s."""
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    L = 2 * math.pi
    g = torch.Generator().manual_seed(7 * n + B)
    u0 = torch.tensor(_rand_u0(B, n, n + B), dtype=torch.float32, device=cuda)
    s0 = 0.05 * (torch.rand(B, n, generator=g) - 0.5).to(cuda)
    nu = (0.005 + 0.02 * torch.rand(B, 1, generator=g)).to(cuda)
    wf = torch.cos(torch.arange(11 * n, device=cuda).reshape(11, n) * 0.01)
    out = []
    for cpt in (1, _WARP_CPT[n]):
        sp = SimpleNamespace(resolution=n, dt=0.2 / n, x=None, adaptive_CFL=None, L=L, nu=nu, device=cuda,
                             convection_term="WENO", equation_type="viscosity", batch_size=B,
                             time_scheme="ssprk3", cells_per_thread=cpt)
        slv = BurgersSolverTorch(sp)
        u = u0.clone().requires_grad_(True)
        s = s0.clone().requires_grad_(True)
        fr = burgers_rollout(slv, u, 11, s=s, ckpt_every=4)
        out.append(torch.autograd.grad((fr * wf).sum(), (u, s)))
    for a, b in zip(*out):
        assert torch.isfinite(a).all()
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 2e-5


@pytest.mark.parametrize("B,n,steps,K,scheme", [
    (3, 64, 1, 1, "ssprk3"), (3, 64, 5, 8, "ssprk3"), (7, 128, 9, 1, "euler"), (7, 128, 17, 16, "ssprk3"),
    (30, 256, 6, 4, "euler"), (60, 128, 13, 5, "ssprk3"), (100, 64, 7, 3, "ssprk3")])
def test_wide_adjoint_segment_corner_cases(cuda, B, n, steps, K, scheme):
    """The small-batch adjoint's forms at segment corner cases (a single step, one
    segment shorter than ckpt_every, ckpt_every = 1, a partial last segment, Euler)
    against the warp-layout adjoint: gradients w.r.t. u0 and s of a frame loss."""
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    L = 2 * math.pi
    g = torch.Generator().manual_seed(B * 1000 + n + steps)
    u0 = torch.tensor(_rand_u0(B, n, B + steps), dtype=torch.float32, device=cuda)
    s0 = 0.05 * (torch.rand(B, n, generator=g) - 0.5).to(cuda)
    wf = torch.randn(B, steps, n, generator=g).to(cuda)
    out = []
    for cpt in (1, _WARP_CPT[n]):
        sp = SimpleNamespace(resolution=n, dt=0.2 / n, x=None, adaptive_CFL=None, L=L, nu=0.01, device=cuda,
                             convection_term="WENO", equation_type="viscosity", batch_size=B,
                             time_scheme=scheme, cells_per_thread=cpt)
        u = u0.clone().requires_grad_(True)
        s = s0.clone().requires_grad_(True)
        fr = burgers_rollout(BurgersSolverTorch(sp), u, steps, s=s, ckpt_every=K)
        out.append(torch.autograd.grad((fr * wf).sum(), (u, s)))
    for a, b in zip(*out):
        assert torch.isfinite(a).all()
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 2e-5


def test_fd_check_fp64_oracle(cuda):
    """GPU adjoint vs FP64 central differences (h=1e-6) of the oracle, 3 SSP-RK3 steps."""
    from inc_b200.solvers import BurgersSolverTorch
    n, B, steps = 64, 3, 3
    p = ob.BurgersParams(resolution=n, L=2 * math.pi, dt=0.01, nu=0.02)
    u0 = _rand_u0(B, n, 21)
    rng = np.random.default_rng(2)
    s0 = 0.1 * rng.standard_normal((B, n))
    w = rng.standard_normal((B, steps, n))
    solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3"))
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    s = torch.tensor(s0, dtype=torch.float32, device=cuda, requires_grad=True)
    solver.correction_s = s
    x, loss = u, 0.0
    wt = torch.tensor(w, dtype=torch.float32, device=cuda)
    for k in range(steps):
        x = solver.step(x)
        loss = loss + (x * wt[:, k]).sum()
    gu, gs = [g.double().cpu().numpy() for g in torch.autograd.grad(loss, (u, s))]

    def L(uu, ss):
        y, t, acc = uu, 0.0, 0.0
        for k in range(steps):
            y, t = ob.step_ssprk3(y, p, t, ss)
            acc += float((y * w[:, k]).sum())
        return acc

    h = 1e-6
    for _ in range(4):
        du, ds = rng.standard_normal(u0.shape), rng.standard_normal(s0.shape)
        fdu = (L(u0 + h * du, s0) - L(u0 - h * du, s0)) / (2 * h)
        fds = (L(u0, s0 + h * ds) - L(u0, s0 - h * ds)) / (2 * h)
        assert abs((gu * du).sum() - fdu) < 1e-4 * max(1.0, abs(fdu))
        assert abs((gs * ds).sum() - fds) < 1e-4 * max(1.0, abs(fds))


def test_ragged_batch_vs_oracle(cuda):
    from inc_b200.batched import RaggedBurgers
    rng = np.random.default_rng(9)
    ns = [64, 512, 128, 256, 64, 8, 32, 256, 128, 16]
    rows = []
    for i, n in enumerate(ns):
        L = 2 * math.pi
        nu = float(np.exp(rng.uniform(np.log(1e-3), np.log(5e-2))))
        u0 = _rand_u0(1, n, 100 + i)[0]
        dx = L / n
        dt = 0.4 * min(dx / np.abs(u0).max(), dx * dx / nu)
        rows.append((u0, nu, dt, dx))
    rb = RaggedBurgers([r[0] for r in rows], [r[1] for r in rows], [r[2] for r in rows], [r[3] for r in rows],
                       scheme="ssprk3", device=cuda)
    out = rb.rollout(steps=25)
    for (u0, nu, dt, dx), got in zip(rows, rb.unpack(out)):
        n = u0.shape[0]
        p = ob.BurgersParams(resolution=n, L=dx * n, dt=dt, nu=nu)
        ref, t = u0[None], 0.0
        for _ in range(25):
            ref, t = ob.step_ssprk3(ref, p, t)
        assert rel_l2(got.cpu().numpy(), ref[0]) < TOL, n


def test_ragged_narrow_rows_share_warps(cuda):
    """Rows narrower than 128 run several per warp (one per lane group); widths mixed so
    that some warps claim rows of another width and run them afterwards."""
    from inc_b200.batched import RaggedBurgers
    rng = np.random.default_rng(21)
    ns = list(rng.choice([8, 16, 32, 64], size=61)) + [128, 256, 512]
    rows = []
    for i, n in enumerate(ns):
        n = int(n)
        nu = float(np.exp(rng.uniform(np.log(1e-3), np.log(5e-2))))
        u0 = _rand_u0(1, n, 300 + i)[0]
        dx = 2 * math.pi / n
        dt = 0.4 * min(dx / np.abs(u0).max(), dx * dx / nu)
        rows.append((u0, nu, dt, dx))
    rb = RaggedBurgers([r[0] for r in rows], [r[1] for r in rows], [r[2] for r in rows], [r[3] for r in rows],
                       scheme="ssprk3", device=cuda)
    out = rb.rollout(steps=12)
    for (u0, nu, dt, dx), got in zip(rows, rb.unpack(out)):
        n = u0.shape[0]
        p = ob.BurgersParams(resolution=n, L=dx * n, dt=dt, nu=nu)
        ref, t = u0[None], 0.0
        for _ in range(12):
            ref, t = ob.step_ssprk3(ref, p, t)
        assert rel_l2(got.cpu().numpy(), ref[0]) < TOL, n


def test_errors(cuda):
    from inc_b200.solvers import BurgersSolverTorch
    p = ob.BurgersParams(resolution=96, L=2 * math.pi, dt=0.01, nu=0.01)
    solver = BurgersSolverTorch(_sim_params(p, 2))
    with pytest.raises(ValueError):
        solver.step(torch.zeros(2, 96, device=cuda))      # n not a power of two
    p2 = ob.BurgersParams(resolution=64, L=2 * math.pi, dt=0.01, nu=0.01, equation_type="cubic")
    with pytest.raises(ValueError):
        BurgersSolverTorch(_sim_params(p2, 2)).step(torch.zeros(2, 64, device=cuda))
    with pytest.raises(TypeError):
        BurgersSolverTorch(_sim_params(ob.BurgersParams(64, 2 * math.pi, 0.01, 0.01), 2)).step(
            torch.zeros(2, 64, device=cuda, dtype=torch.float64))


def test_nonfinite_propagates(cuda):
    from inc_b200.solvers import BurgersSolverTorch
    p = ob.BurgersParams(resolution=64, L=2 * math.pi, dt=0.01, nu=0.01)
    solver = BurgersSolverTorch(_sim_params(p, 3))
    u = torch.zeros(3, 64, device=cuda)
    u[1, 7] = float("nan")
    out = solver.step(u)
    assert torch.isnan(out[1]).any() and torch.isfinite(out[0]).all() and torch.isfinite(out[2]).all()


def test_step_descriptor_cache_follows_parameters(cuda):
    """step() reuses its launch descriptor across calls: a parameter modified in place or
    replaced, and the time of a forcing ('learning') step under autograd, must still reach
    the kernel exactly as a freshly built descriptor would pass them."""
    from inc_b200.solvers import BurgersSolverTorch, BurgersStepFn
    B, n = 5, 64
    rng = np.random.default_rng(21)
    p = ob.BurgersParams(resolution=n, L=2 * math.pi, dt=0.01, nu=rng.uniform(0.005, 0.05, (B, 1)),
                         equation_type="learning", A=rng.uniform(-0.5, 0.5, (B, 1, 3)),
                         omega=rng.uniform(-0.4, 0.4, (B, 1, 3)), phi=rng.uniform(0, 6.28, (B, 1, 3)),
                         l=rng.integers(1, 4, (B, 1, 3)).astype(np.float64), x=np.arange(n) * (2 * math.pi / n))
    sp = _sim_params(p, B, "ssprk3")
    solver = BurgersSolverTorch(sp)
    solver.t = torch.tensor(rng.uniform(0, 1, (B, 1)), dtype=torch.float32, device=cuda)
    u0 = torch.tensor(_rand_u0(B, n, 8), dtype=torch.float32, device=cuda)

    def fresh_step(u, t):
        launch = solver.launch_for(u, t)
        out = torch.empty_like(u)
        launch.step(u, None, out)
        return out

    t0 = solver.t.clone()
    a = solver.step(u0)
    assert torch.equal(a, fresh_step(u0, t0))
    sp.nu.mul_(2.0)                      # in place: same tensor object, new version
    t1 = solver.t.clone()
    b = solver.step(u0)
    assert torch.equal(b, fresh_step(u0, t1)) and not torch.equal(a, b)
    sp.A = sp.A * 0.5                    # replaced by a new tensor
    t2 = solver.t.clone()
    c = solver.step(u0)
    assert torch.equal(c, fresh_step(u0, t2)) and not torch.equal(b, c)
    # autograd over three cached steps while solver.t advances in place: the backward of each
    # step sees that step's time
    u = u0.clone().requires_grad_(True)
    solver.t = t0.clone()
    x, ts = u, []
    for _ in range(3):
        ts.append(solver.t.clone())
        x = solver.step(x)
    w = torch.randn_like(x)
    g_cached, = torch.autograd.grad((x * w).sum(), (u,))
    u2 = u0.clone().requires_grad_(True)
    y = u2
    for t in ts:
        y = BurgersStepFn.apply(y, None, solver.launch_for(y, t))
    g_fresh, = torch.autograd.grad((y * w).sum(), (u2,))
    assert torch.equal(x, y) and torch.equal(g_cached, g_fresh)
