"""KS CUDA path vs the FP64 oracle and the reference's golden vectors (GPU).

Tolerance: relative L2 <= 1e-5 against FP64 within the stated horizon (the KS
system is chaotic; FP32 and FP64 trajectories decorrelate after ~80 step()
calls, so long rollouts are checked against an FP32 run of the same maths).
"""
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import ks as oks
from tests.golden_io import ks_case, load, rel_l2

pytestmark = pytest.mark.gpu
KZ = load("ks_golden.npz")
TOL = 1e-5


def _solver(N, dt, scheme="ETRK2", Ls=None, tpp=0, dealias=False, device="cuda"):
    from inc_b200.solvers import KSSolverTorch
    ds = torch.tensor(Ls if Ls is not None else [64.0], dtype=torch.float32, device=device)
    sp = SimpleNamespace(resolution=N, dt=dt, device=device, domain_size=ds, alpha=torch.zeros_like(ds),
                         time_scheme=scheme, threads_per_pair=tpp, dealias=dealias)
    return KSSolverTorch(sp)


def _u0(B, N, Ls, seed):
    from inc_b200.workloads import ks_u0
    rng = np.random.default_rng(seed)
    return np.stack([ks_u0(rng, 1, N, L)[0] for L in Ls])


@pytest.mark.parametrize("name", [str(n) for n in KZ["cases"]])
def test_golden_steps(cuda, name):
    c = ks_case(KZ, name)
    frames = KZ[f"{name}.frames"]
    solver = _solver(c["N"], c["dt"], c["scheme"], list(c["L"]))
    ds = torch.tensor(c["L"], dtype=torch.float32, device=cuda)
    f = lambda a: None if a is None else torch.tensor(a, dtype=torch.float32, device=cuda)  # noqa: E731
    solver.correction_s, solver.correction_u = f(c["s"]), f(c["cu"])
    u = f(c["u0"])
    for k in range(frames.shape[1]):
        u = solver.step(u, ds)
        assert rel_l2(u.cpu().numpy(), frames[:, k]) < TOL, (name, k)


@pytest.mark.parametrize("N,tpp", [(16, 4), (32, 8), (64, 16), (64, 8), (128, 32), (128, 16), (256, 64), (256, 32),
                                   (256, 16), (512, 64), (512, 32), (512, 16)])
@pytest.mark.parametrize("mixed", [False, True])
def test_shapes_vs_oracle(cuda, N, tpp, mixed):
    B = 7  # odd: one lone row
    Ls = [50.0 + 7.0 * i for i in range(B)] if mixed else [64.0] * B
    u0 = _u0(B, N, Ls, N)
    rng = np.random.default_rng(1)
    s = 0.01 * rng.standard_normal((B, N))
    dt = 0.1
    solver = _solver(N, dt, "ETRK2", Ls, tpp)
    solver.correction_s = torch.tensor(s, dtype=torch.float32, device=cuda)
    ds = torch.tensor(Ls, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    coeffs = oks.coefficients_fp64(Ls, N, dt, "ETRK2", np.float64)
    ref = u0
    for _ in range(10):
        u = solver.step(u, ds)
        ref = oks.step(ref, Ls, dt, "ETRK2", s, None, coeffs)
    assert rel_l2(u.cpu().numpy(), ref) < TOL


def test_etd1_small_dt(cuda):
    N, B, dt = 64, 6, 0.05
    Ls = [32.0, 32.0, 40.0, 40.0, 22.0, 64.0]
    u0 = _u0(B, N, Ls, 4)
    solver = _solver(N, dt, "ETD1", Ls)
    ds = torch.tensor(Ls, dtype=torch.float32, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda)
    ref = u0
    for _ in range(20):
        u = solver.step(u, ds)
        ref = oks.step(ref, Ls, dt, "ETD1")
    assert rel_l2(u.cpu().numpy(), ref) < TOL


def test_config1_horizon(cuda):
    """KS plain config (L=64, N=256, dt=0.25, ETRK2, seeded s) at 1, 10, 20 step() calls."""
    from inc_b200.workloads import ks_plain_config
    cfg = ks_plain_config(B=128)
    N, L, dt = cfg["N"], cfg["L"], cfg["dt"]
    solver = _solver(N, dt, "ETRK2", [L] * cfg["B"])
    solver.correction_s = torch.tensor(cfg["s"], dtype=torch.float32, device=cuda)
    ds = torch.full((cfg["B"],), L, device=cuda)
    u = torch.tensor(cfg["u0"], dtype=torch.float32, device=cuda)
    ref = cfg["u0"]
    errs = {}
    for k in range(1, 21):
        u = solver.step(u, ds)
        ref = oks.step(ref, [L] * cfg["B"], dt, "ETRK2", cfg["s"])
        if k in (1, 10, 20):
            errs[k] = rel_l2(u.cpu().numpy(), ref)
    assert all(e < TOL for e in errs.values()), errs


def test_fused_rollout_matches_steps(cuda):
    from inc_b200.rollout import ks_rollout
    N, B, dt = 256, 10, 0.25
    Ls = [64.0] * 6 + [48.0] * 4
    u0 = torch.tensor(_u0(B, N, Ls, 7), dtype=torch.float32, device=cuda)
    s = 0.01 * torch.randn(B, N, device=cuda)
    ds = torch.tensor(Ls, device=cuda)
    a = _solver(N, dt, "ETRK2", Ls)
    a.correction_s = s
    u, frames = u0, []
    for _ in range(20):
        u = a.step(u, ds)
        frames.append(u)
    b = _solver(N, dt, "ETRK2", Ls)
    fused = ks_rollout(b, u0, 20, ds, s=s).cpu().numpy()
    # The fused launch carries the spectrum across steps while a step() call
    # re-transforms u at each step start: the two differ by rounding, which the
    # chaotic dynamics amplify.  Both must sit within 1e-5 of FP64 at 20 steps.
    ref, sn = u0.cpu().numpy().astype(np.float64), s.cpu().numpy().astype(np.float64)
    for k in range(20):
        ref = oks.step(ref, Ls, dt, "ETRK2", sn)
        assert rel_l2(fused[:, k], ref) < TOL, k
        assert rel_l2(frames[k].cpu().numpy(), ref) < TOL, k


@pytest.mark.parametrize("name", [str(n) for n in KZ["grad_cases"]])
def test_step_gradients_vs_reference_autograd(cuda, name):
    c = ks_case(KZ, name)
    w = torch.tensor(KZ[f"{name}.w"], dtype=torch.float32, device=cuda)
    solver = _solver(c["N"], c["dt"], c["scheme"], list(c["L"]))
    ds = torch.tensor(c["L"], dtype=torch.float32, device=cuda)
    u = torch.tensor(c["u0"], dtype=torch.float32, device=cuda, requires_grad=True)
    s = torch.tensor(c["s"], dtype=torch.float32, device=cuda, requires_grad=True)
    solver.correction_s = s
    x, loss = u, 0.0
    for k in range(w.shape[1]):
        x = solver.step(x, ds)
        loss = loss + (x * w[:, k]).sum()
    gu, gs = torch.autograd.grad(loss, (u, s))
    assert rel_l2(gu.cpu().numpy(), KZ[f"{name}.grad_u"]) < 1e-4
    assert rel_l2(gs.cpu().numpy(), KZ[f"{name}.grad_s"]) < 1e-4


def test_correction_u_gradient(cuda):
    N, B = 32, 4
    Ls = [30.0, 30.0, 40.0, 44.0]
    solver = _solver(N, 0.1, "ETRK2", Ls)
    ds = torch.tensor(Ls, device=cuda)
    u = torch.tensor(_u0(B, N, Ls, 3), dtype=torch.float32, device=cuda, requires_grad=True)
    cu = (0.01 * torch.randn(B, N, device=cuda)).requires_grad_(True)
    solver.correction_u = cu
    out = solver.step(u, ds)
    w = torch.randn_like(out)
    gu, gcu = torch.autograd.grad((out * w).sum(), (u, cu))
    assert torch.equal(gu, gcu)


@pytest.mark.parametrize("mixed", [False, True])
def test_rollout_backward_matches_stepwise(cuda, mixed):
    from inc_b200.rollout import ks_rollout
    N, B, dt, steps = 128, 6, 0.2, 13
    Ls = [40.0, 44.0, 50.0, 60.0, 64.0, 100.0] if mixed else [64.0] * B
    u0 = torch.tensor(_u0(B, N, Ls, 11), dtype=torch.float32, device=cuda)
    s0 = 0.01 * torch.randn(B, N, device=cuda)
    w = torch.randn(B, steps, N, device=cuda)
    ds = torch.tensor(Ls, device=cuda)
    a = _solver(N, dt, "ETRK2", Ls)
    u, s = u0.clone().requires_grad_(True), s0.clone().requires_grad_(True)
    a.correction_s = s
    x, frames = u, []
    for _ in range(steps):
        x = a.step(x, ds)
        frames.append(x)
    ga = torch.autograd.grad((torch.stack(frames, 1) * w).sum(), (u, s))
    b = _solver(N, dt, "ETRK2", Ls)
    u2, s2 = u0.clone().requires_grad_(True), s0.clone().requires_grad_(True)
    fr = ks_rollout(b, u2, steps, ds, s=s2, ckpt_every=4)
    gb = torch.autograd.grad((fr * w).sum(), (u2, s2))
    for x1, x2 in zip(ga, gb):
        assert rel_l2(x2.cpu().numpy(), x1.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("N,tpp", [(16, 4), (64, 16), (128, 32), (256, 32), (256, 64), (512, 32)])
@pytest.mark.parametrize("scheme", ["ETRK2", "ETD1"])
def test_rollout_backward_scratch_matches_rebuild(cuda, N, tpp, scheme):
    """The rollout backward that keeps the segment replay's substep states in
    device scratch against the one that rebuilds them per step: odd batch (a
    lone row), a short last segment, frame and final-state adjoints."""
    B, steps, K = 7, 11, 4
    dt = 0.2 if scheme == "ETRK2" else 0.05
    Ls = [40.0 + 9 * i for i in range(B)]
    solver = _solver(N, dt, scheme, Ls, tpp=tpp)
    u0 = torch.tensor(_u0(B, N, Ls, 5), dtype=torch.float32, device=cuda)
    g = torch.Generator(device=cuda).manual_seed(N + tpp)
    s = 0.01 * torch.randn(B, N, device=cuda, generator=g)
    ds = torch.tensor(Ls, device=cuda)
    plan = solver.plan_for(u0, ds)
    frames = torch.empty(B, steps, N, device=cuda)
    ck = torch.empty(B, (steps + K - 1) // K, N, device=cuda)
    plan.rollout(u0, s, steps, frames, None, K, ck)
    gf = torch.randn(B, steps, N, device=cuda, generator=g)
    gfin = torch.randn(B, N, device=cuda, generator=g)
    out = []
    for work in (None, False):
        gu, gs = torch.empty_like(u0), torch.empty_like(u0)
        plan.rollout_bwd(ck, s, steps, K, gf, gfin, gu, gs, work=work)
        out.append((gu, gs))
    for a, b in zip(*out):
        assert torch.isfinite(a).all()
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5
    small = torch.empty(plan.rollout_bwd_work_size(K) - 16, dtype=torch.uint8, device=cuda)
    with pytest.raises((ValueError, RuntimeError)):
        plan.rollout_bwd(ck, s, steps, K, gf, gfin, gu, gs, work=small)


@pytest.mark.parametrize("N,B,steps,K", [(256, 7, 1, 4), (256, 5, 3, 4), (256, 9, 11, 4), (256, 3, 9, 1),
                                          (128, 11, 13, 8)])
def test_rollout_backward_two_warp_form(cuda, N, B, steps, K):
    """The checkpointed backward with its replay on a second warp (32 lanes, ETRK2, one
    domain size per pair) against the one-warp rebuilding form: a single step, one
    segment shorter than ckpt_every, ckpt_every = 1, partial last segments, a lone row."""
    dt = 0.2
    Ls = [56.0] * B
    solver = _solver(N, dt, "ETRK2", Ls, tpp=32)
    u0 = torch.tensor(_u0(B, N, Ls, 9), dtype=torch.float32, device=cuda)
    g = torch.Generator(device=cuda).manual_seed(N + B + steps)
    s = 0.01 * torch.randn(B, N, device=cuda, generator=g)
    ds = torch.tensor(Ls, device=cuda)
    plan = solver.plan_for(u0, ds)
    frames = torch.empty(B, steps, N, device=cuda)
    ck = torch.empty(B, (steps + K - 1) // K, N, device=cuda)
    plan.rollout(u0, s, steps, frames, None, K, ck)
    gf = torch.randn(B, steps, N, device=cuda, generator=g)
    gfin = torch.randn(B, N, device=cuda, generator=g)
    out = []
    for work in (None, False):
        gu, gs = torch.empty_like(u0), torch.empty_like(u0)
        plan.rollout_bwd(ck, s, steps, K, gf, gfin, gu, gs, work=work)
        out.append((gu, gs))
    for a, b in zip(*out):
        assert torch.isfinite(a).all()
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("B,tpp", [(1031, 16), (4101, 32)])
def test_rollout_backward_scratch_many_groups(cuda, B, tpp):
    """The scratch backward on grids of many blocks with several row pairs per block
    and a partial last block (odd B: a lone row too), against the rebuilding form:
    each launched group's scratch slot and the padding of the scratch size."""
    N, steps, K, dt = 256, 11, 4, 0.25
    Ls = [64.0] * B
    solver = _solver(N, dt, "ETRK2", Ls, tpp=tpp)
    from inc_b200.workloads import ks_plain_config
    cfg = ks_plain_config(B=B, steps=steps)
    u0 = torch.tensor(cfg["u0"], dtype=torch.float32, device=cuda)
    s = torch.tensor(cfg["s"], dtype=torch.float32, device=cuda)
    ds = torch.full((B,), 64.0, device=cuda)
    plan = solver.plan_for(u0, ds)
    frames = torch.empty(B, steps, N, device=cuda)
    ck = torch.empty(B, (steps + K - 1) // K, N, device=cuda)
    plan.rollout(u0, s, steps, frames, None, K, ck)
    g = torch.Generator(device=cuda).manual_seed(B)
    gf = torch.randn(B, steps, N, device=cuda, generator=g)
    out = []
    for work in (None, False):
        gu, gs = torch.empty_like(u0), torch.empty_like(u0)
        plan.rollout_bwd(ck, s, steps, K, gf, None, gu, gs, work=work)
        out.append((gu.cpu().numpy(), gs.cpu().numpy()))
    for a, b in zip(*out):
        assert np.isfinite(a).all()
        assert rel_l2(a, b) < 1e-5
        # row by row: no row's slot was shared or skipped
        per_row = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
        assert per_row.max() < 1e-4


@pytest.mark.parametrize("N,tpp,B", [(16, 4, 7), (64, 16, 7), (128, 32, 7), (256, 32, 7), (256, 64, 7),
                                     (512, 32, 7), (256, 32, 1031), (256, 16, 4101)])
@pytest.mark.parametrize("scheme", ["ETRK2", "ETD1"])
def test_rollout_tape_matches_checkpointed(cuda, N, tpp, B, scheme):
    """The tape rollout (every step's states recorded, no replay in the backward) against
    the checkpointed rollout and its scratch backward: the same frames bit for bit, and
    gradients (u0, s; frame and final-state adjoints) equal to rounding."""
    steps, K = 11, 4
    dt = 0.2 if scheme == "ETRK2" else 0.05
    Ls = [40.0 + 9 * (i % 7) for i in range(B)]
    solver = _solver(N, dt, scheme, Ls, tpp=tpp)
    u0 = torch.tensor(_u0(B, N, Ls, 5) if B < 100 else np.tile(_u0(7, N, Ls[:7], 5), (B // 7 + 1, 1))[:B],
                      dtype=torch.float32, device=cuda)
    g = torch.Generator(device=cuda).manual_seed(N + tpp + B)
    s = 0.01 * torch.randn(B, N, device=cuda, generator=g)
    ds = torch.tensor(Ls, device=cuda)
    plan = solver.plan_for(u0, ds)
    fa = torch.empty(B, steps, N, device=cuda)
    ck = torch.empty(B, (steps + K - 1) // K, N, device=cuda)
    plan.rollout(u0, s, steps, fa, None, K, ck)
    fb = torch.empty(B, steps, N, device=cuda)
    tape = torch.empty(plan.tape_size(steps), dtype=torch.uint8, device=cuda)
    plan.rollout_tape(u0, s, steps, fb, None, tape)
    assert torch.equal(fa, fb)
    gf = torch.randn(B, steps, N, device=cuda, generator=g)
    gfin = torch.randn(B, N, device=cuda, generator=g)
    ga = [torch.empty_like(u0) for _ in range(2)]
    gb = [torch.empty_like(u0) for _ in range(2)]
    plan.rollout_bwd(ck, s, steps, K, gf, gfin, ga[0], ga[1])
    plan.rollout_bwd_tape(tape, s, steps, gf, gfin, gb[0], gb[1])
    for a, b in zip(ga, gb):
        assert torch.isfinite(b).all()
        assert rel_l2(b.cpu().numpy(), a.cpu().numpy()) < 1e-5
    with pytest.raises(ValueError):
        plan.rollout_bwd_tape(tape[:-16], s, steps, gf, gfin, gb[0], gb[1])


def test_ks_rollout_tape_autograd(cuda):
    from inc_b200.rollout import ks_rollout
    N, B, steps, dt = 128, 6, 9, 0.2
    Ls = [40.0, 44.0, 50.0, 60.0, 64.0, 100.0]
    u0 = torch.tensor(_u0(B, N, Ls, 13), dtype=torch.float32, device=cuda)
    s0 = 0.01 * torch.randn(B, N, device=cuda)
    w = torch.randn(B, steps, N, device=cuda)
    ds = torch.tensor(Ls, device=cuda)
    out = []
    for k in (4, 0):
        u, s = u0.clone().requires_grad_(True), s0.clone().requires_grad_(True)
        fr = ks_rollout(_solver(N, dt, "ETRK2", Ls), u, steps, ds, s=s, ckpt_every=k)
        out.append(torch.autograd.grad((fr * w).sum(), (u, s)))
    for a, b in zip(*out):
        assert rel_l2(b.cpu().numpy(), a.cpu().numpy()) < 1e-5


def test_fd_check_fp64_oracle(cuda):
    N, B, dt, steps = 64, 3, 0.25, 2
    Ls = [64.0, 64.0, 50.0]
    u0 = _u0(B, N, Ls, 5)
    rng = np.random.default_rng(6)
    s0 = 0.01 * rng.standard_normal((B, N))
    w = rng.standard_normal((B, steps, N))
    solver = _solver(N, dt, "ETRK2", Ls)
    ds = torch.tensor(Ls, device=cuda)
    u = torch.tensor(u0, dtype=torch.float32, device=cuda, requires_grad=True)
    s = torch.tensor(s0, dtype=torch.float32, device=cuda, requires_grad=True)
    solver.correction_s = s
    x, loss = u, 0.0
    wt = torch.tensor(w, dtype=torch.float32, device=cuda)
    for k in range(steps):
        x = solver.step(x, ds)
        loss = loss + (x * wt[:, k]).sum()
    gu, gs = [g.double().cpu().numpy() for g in torch.autograd.grad(loss, (u, s))]

    def L(uu, ss):
        y, acc = uu, 0.0
        for k in range(steps):
            y = oks.step(y, Ls, dt, "ETRK2", ss)
            acc += float((y * w[:, k]).sum())
        return acc

    h = 1e-6
    for _ in range(4):
        du, dss = rng.standard_normal(u0.shape), rng.standard_normal(s0.shape)
        fdu = (L(u0 + h * du, s0) - L(u0 - h * du, s0)) / (2 * h)
        fds = (L(u0, s0 + h * dss) - L(u0, s0 - h * dss)) / (2 * h)
        assert abs((gu * du).sum() - fdu) < 1e-4 * max(1.0, abs(fdu))
        assert abs((gs * dss).sum() - fds) < 1e-4 * max(1.0, abs(fds))


def test_dealias_option_truncates_nonlinear_term(cuda):
    """The opt-in 2/3 rule: the nonlinear term has no modes with 3|k| > N."""
    N, B = 64, 2
    Ls = [64.0, 64.0]
    solver = _solver(N, 0.05, "ETD1", Ls, dealias=True)
    ds = torch.tensor(Ls, device=cuda)
    u0 = _u0(B, N, Ls, 9)
    u = solver.step(torch.tensor(u0, dtype=torch.float32, device=cuda), ds).cpu().numpy()
    # reference-style update with a 2/3-truncated nonlinear term
    lop, wn = oks.linear_operator(Ls, N)
    e, p1, _ = oks.etd_coefficients(lop, 0.05, "ETD1")
    f = np.fft.fftfreq(N) * N
    mask = (3 * np.abs(f) <= N).astype(float)
    y = u0
    for _ in range(2):
        nh = -0.5 * wn * np.fft.fft(y * y) * mask
        y = np.fft.ifft(e * np.fft.fft(y) + p1 * nh).real
    assert rel_l2(u, y) < TOL


def test_errors(cuda):
    from inc_b200.solvers import KSSolverTorch
    with pytest.raises(KeyError):
        KSSolverTorch(SimpleNamespace(resolution=64, dt=0.1, device="cuda", domain_size=torch.ones(2),
                                      alpha=torch.zeros(2), time_scheme="RK4"))
    solver = _solver(96, 0.1)
    with pytest.raises(ValueError):
        solver.step(torch.zeros(2, 96, device=cuda), torch.tensor([64.0, 64.0], device=cuda))
    solver = _solver(64, 0.1)
    with pytest.raises(ValueError):
        solver.step(torch.zeros(2, 64, device=cuda), torch.tensor([64.0, -1.0], device=cuda))
