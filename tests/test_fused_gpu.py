"""Burgers rollout with the periodic CNN corrector inside the kernel (GPU).

The fused kernel (inc_burgers_cnn_rollout) must reproduce the per-step loop
of simulate_rollout (trainer_1d.py:154-183): s = model(u); u = step(u, s).
Checked against (a) that loop in FP64 on the CPU (torch's Conv1d in float64
plus the oracle's Burgers step) and (b) the same loop on the GPU in FP32
(cuDNN convolutions with TF32 off plus the CUDA solver), over all supported
widths, both time schemes, both convection schemes and the reference's
source terms, with batches that leave the last CTA partly empty."""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import burgers as ob
from tests.golden_io import burgers_case, load, rel_l2

pytestmark = pytest.mark.gpu
BZ = load("burgers_golden.npz")
TOL = 1e-5  # relative L2 of FP32 vs FP64 frames / corrections


@pytest.fixture(autouse=True)
def fp32_convs():
    saved = (torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32)
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    yield
    torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = saved


def _params(N, eq="viscosity", conv="WENO", B=1, seed=0):
    rng = np.random.default_rng(seed)
    L = 2 * math.pi
    kw = dict(resolution=N, L=L, dt=0.25 * L / N / 1.5, nu=0.01, convection_term=conv, equation_type=eq)
    if eq == "linear":
        kw["beta"] = 0.1
    if eq == "learning":
        J = 3
        kw.update(A=rng.uniform(-0.5, 0.5, (B, 1, J)), omega=rng.uniform(-0.4, 0.4, (B, 1, J)),
                  phi=rng.uniform(0, 2 * np.pi, (B, 1, J)), l=rng.integers(1, 4, (B, 1, J)).astype(np.float64),
                  x=np.arange(N) * (L / N))
    return ob.BurgersParams(**kw)


def _sim_params(p, B, scheme, device):
    f = lambda a: None if a is None else torch.as_tensor(a, dtype=torch.float32, device=device)  # noqa: E731
    arr = lambda a: f(a) if isinstance(a, np.ndarray) else a  # noqa: E731
    return SimpleNamespace(resolution=p.resolution, dt=p.dt, x=f(p.x) if p.x is not None else None,
                           adaptive_CFL=None, L=p.L, nu=arr(p.nu), device=device, convection_term=p.convection_term,
                           equation_type=p.equation_type, batch_size=B,
                           beta=arr(p.beta), J=(p.A.shape[-1] if p.A is not None else 0), A=f(p.A),
                           omega=f(p.omega), phi=f(p.phi), l=f(p.l), time_scheme=scheme)


def _u0(B, N, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(N) * (2 * np.pi / N)
    a = rng.uniform(-0.5, 0.5, (B, 5))
    ph = rng.uniform(0, 2 * np.pi, (B, 5))
    k = np.arange(1, 6)
    return (a[:, :, None] * np.sin(k[None, :, None] * x[None, None, :] + ph[:, :, None])).sum(1)


def _net(seed=0):
    from inc_b200.correctors import PeriodicCNN1D
    torch.manual_seed(seed)
    net = PeriodicCNN1D()
    with torch.no_grad():  # larger corrections than the default init, so that s matters
        for c in net.convs:
            c.weight.mul_(3.0)
    return net


def _fp64_loop(net, p, u0, steps, scheme, t0=0.0):
    """The per-step loop in float64 on the CPU: torch corrector + oracle step."""
    net64 = net.double().cpu()
    u, t = u0.astype(np.float64), t0
    frames, corr = [], []
    with torch.no_grad():
        for _ in range(steps):
            s = net64(torch.from_numpy(u)).numpy()
            u, t = (ob.step_ssprk3 if scheme == "ssprk3" else ob.step_euler)(u, p, t, s)
            frames.append(u)
            corr.append(s)
    return np.stack(frames, 1), np.stack(corr, 1)


@pytest.mark.parametrize("N,B", [(64, 3), (128, 5), (256, 7), (512, 2)])
@pytest.mark.parametrize("scheme", ["euler", "ssprk3"])
def test_fused_cnn_rollout_vs_fp64_loop(cuda, N, B, scheme):
    from inc_b200.fused import burgers_cnn_rollout
    from inc_b200.solvers import BurgersSolverTorch
    p = _params(N)
    u0 = _u0(B, N, seed=N + B)
    net = _net()
    steps = 12
    ref_f, ref_c = _fp64_loop(net, p, u0, steps, scheme)
    solver = BurgersSolverTorch(_sim_params(p, B, scheme, cuda))
    with torch.no_grad():
        frames, corr = burgers_cnn_rollout(net.float().to(cuda), solver,
                                           torch.tensor(u0, dtype=torch.float32, device=cuda), steps)
    assert rel_l2(frames.cpu().numpy(), ref_f) < TOL
    assert rel_l2(corr.cpu().numpy(), ref_c) < TOL
    assert np.max(np.abs(corr.cpu().numpy())) > 1e-2  # the corrector is not negligible
    assert abs(float(solver.t) - steps * p.dt) < 1e-9


@pytest.mark.parametrize("eq,conv", [("viscosity", "FDM"), ("linear", "WENO"), ("learning", "WENO"),
                                     ("homogeneous", "WENO")])
def test_fused_cnn_rollout_sources_and_convection(cuda, eq, conv):
    from inc_b200.fused import burgers_cnn_rollout
    from inc_b200.solvers import BurgersSolverTorch
    N, B, steps = 128, 9, 10
    p = _params(N, eq=eq, conv=conv, B=B, seed=1)
    u0 = _u0(B, N, seed=3)
    net = _net(1)
    ref_f, ref_c = _fp64_loop(net, p, u0, steps, "ssprk3", t0=0.3)
    solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
    solver.t = 0.3
    with torch.no_grad():
        frames, corr = burgers_cnn_rollout(net.float().to(cuda), solver,
                                           torch.tensor(u0, dtype=torch.float32, device=cuda), steps)
    assert rel_l2(frames.cpu().numpy(), ref_f) < TOL
    assert rel_l2(corr.cpu().numpy(), ref_c) < TOL


def _per_step_loop(net, solver, u0, steps):
    """The reference's loop on the GPU: torch corrector + one CUDA step() per step."""
    u, frames, corr = u0, [], []
    for _ in range(steps):
        c = net(u)
        solver.correction_s = c
        u = solver.step(u)
        frames.append(u)
        corr.append(c)
    return torch.stack(frames, 1), torch.stack(corr, 1)


def test_fused_matches_per_step_gpu_loop_and_dispatch(cuda):
    """simulate_rollout takes the fused kernel with gradients off and on; both match the loop."""
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch
    N, B, steps = 256, 37, 16
    p = _params(N)
    u0 = torch.tensor(_u0(B, N, seed=5), dtype=torch.float32, device=cuda)
    net = _net(2).float().to(cuda)
    s1 = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
    with torch.no_grad():
        f1, c1 = simulate_rollout(net, s1, u0, steps, "INC")
    s2 = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
    f2, c2 = simulate_rollout(net, s2, u0, steps, "INC")  # grad enabled: fused training path
    assert f2.requires_grad and f2.grad_fn is not None
    s3 = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
    with torch.no_grad():
        f3, c3 = _per_step_loop(net, s3, u0, steps)
    for f, c in ((f1, c1), (f2.detach(), c2.detach())):
        assert rel_l2(f.cpu().numpy(), f3.cpu().numpy()) < TOL
        assert rel_l2(c.cpu().numpy(), c3.cpu().numpy()) < TOL
    assert abs(float(s1.t) - float(s2.t)) < 1e-9 and abs(float(s1.t) - float(s3.t)) < 1e-9
    assert torch.equal(s1.correction_s, c1[:, -1])


@pytest.mark.parametrize("N,B,scheme,K,eq", [
    (256, 5, "ssprk3", 8, "viscosity"), (256, 5, "ssprk3", 5, "learning"), (256, 5, "euler", 1, "linear"),
    (256, 5, "ssprk3", 32, "viscosity"),
    # four rows per CTA at n = 64 and two at n = 128: batches that leave the last CTA partly empty
    (64, 9, "ssprk3", 8, "viscosity"), (64, 6, "euler", 1, "linear"), (128, 5, "ssprk3", 5, "learning"),
    (128, 4, "ssprk3", 13, "viscosity"),
    # one CTA of 512 threads per row; 26 is the longest segment that fits beside the activations
    (512, 3, "ssprk3", 8, "viscosity"), (512, 2, "ssprk3", 26, "learning")])
def test_fused_training_gradients_vs_per_step_loop(cuda, N, B, scheme, K, eq):
    """Gradients of a loss on frames and corrections w.r.t. u0 and every network parameter:
    fused backward (segment replay, recomputed activations) vs torch autograd through the loop,
    at every supported row width."""
    from inc_b200.fused import burgers_cnn_rollout
    from inc_b200.solvers import BurgersSolverTorch
    steps = 13 if K <= 13 else K + 3
    p = _params(N, eq=eq, B=B, seed=6)
    u0_np = _u0(B, N, seed=7)
    gen = torch.Generator().manual_seed(3)
    wf = torch.randn(B, steps, N, generator=gen).to(cuda)
    wc = torch.randn(B, steps, N, generator=gen).to(cuda)

    def run(fused):
        net = _net(5).float().to(cuda)
        solver = BurgersSolverTorch(_sim_params(p, B, scheme, cuda))
        solver.t = 0.2
        u0 = torch.tensor(u0_np, dtype=torch.float32, device=cuda, requires_grad=True)
        if fused:
            f, c = burgers_cnn_rollout(net, solver, u0, steps, ckpt_every=K)
        else:
            f, c = _per_step_loop(net, solver, u0, steps)
        loss = (f * wf).sum() + 3.0 * (c * wc).sum()
        loss.backward()
        return loss.item(), u0.grad.cpu().numpy(), [q.grad.cpu().numpy() for q in net.parameters()]

    lf, gf, pf = run(True)
    lr, gr, pr = run(False)
    assert abs(lf - lr) <= 1e-5 * max(1.0, abs(lr))
    assert rel_l2(gf, gr) < 1e-4
    for a, b in zip(pf, pr):
        assert rel_l2(a, b) < 1e-4
    assert max(np.abs(b).max() for b in pr) > 0


@pytest.mark.parametrize("N,B", [(64, 9), (256, 5), (512, 2)])
def test_fused_training_recorded_activations_match_recompute(cuda, monkeypatch, N, B):
    """The training path keeps the hidden layers' pre-activations from the forward
    (inc_burgers_cnn_rollout_acts / _bwd_acts) when they fit, else the backward
    recomputes them from the replayed states: the two agree (the record holds the
    forward's own states, the replay its recomputation, equal to FP32 rounding)."""
    from inc_b200 import fused
    from inc_b200.solvers import BurgersSolverTorch
    steps = 11
    p = _params(N, B=B, seed=13)
    u0_np = _u0(B, N, seed=14)
    gen = torch.Generator().manual_seed(5)
    wf = torch.randn(B, steps, N, generator=gen).to(cuda)
    wc = torch.randn(B, steps, N, generator=gen).to(cuda)

    def run(acts_max):
        monkeypatch.setattr(fused, "ACTS_BYTES_MAX", acts_max)
        net = _net(3).float().to(cuda)
        solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
        u0 = torch.tensor(u0_np, dtype=torch.float32, device=cuda, requires_grad=True)
        f, c = fused.burgers_cnn_rollout(net, solver, u0, steps, ckpt_every=4)
        ((f * wf).sum() + (c * wc).sum()).backward()
        return [u0.grad.cpu().numpy()] + [q.grad.cpu().numpy() for q in net.parameters()]

    rec, recomp = run(4 << 30), run(0)
    for a, b in zip(rec, recomp):
        assert np.isfinite(a).all()
        assert rel_l2(a, b) < 1e-5


def test_fused_training_frames_only_loss_and_graph_capture(cuda):
    """A loss on the frames alone (the corrections' adjoint is zero) and the whole training
    step (fused forward + backward + optimizer) replayed from a CUDA graph."""
    from inc_b200.fused import burgers_cnn_rollout
    from inc_b200.solvers import BurgersSolverTorch
    N, B, steps = 256, 6, 10
    p = _params(N)
    u0 = torch.tensor(_u0(B, N, seed=9), dtype=torch.float32, device=cuda)
    target = torch.zeros(B, steps, N, device=cuda)
    grads = []
    for fused in (True, False):
        net = _net(6).float().to(cuda)
        solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
        f, _ = (burgers_cnn_rollout(net, solver, u0, steps, ckpt_every=4) if fused
                else _per_step_loop(net, solver, u0, steps))
        torch.mean((f - target) ** 2).backward()
        grads.append([q.grad.clone() for q in net.parameters()])
    for a, b in zip(*grads):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-4
    # graph capture of the training step
    net = _net(6).float().to(cuda)
    solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
    opt = torch.optim.SGD(net.parameters(), lr=1e-3)

    def train_step():
        solver.t = 0.0
        f, _ = burgers_cnn_rollout(net, solver, u0, steps, ckpt_every=4)
        torch.mean((f - target) ** 2).backward()
        opt.step()
        opt.zero_grad(set_to_none=False)

    side = torch.cuda.Stream(cuda)
    side.wait_stream(torch.cuda.current_stream(cuda))
    with torch.cuda.stream(side):
        for _ in range(2):
            train_step()
    torch.cuda.current_stream(cuda).wait_stream(side)
    w_before = net.convs[1].weight.detach().clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        train_step()
    graph.replay()
    torch.cuda.synchronize()
    assert not torch.equal(net.convs[1].weight.detach(), w_before)
    assert torch.isfinite(net.convs[1].weight).all()


def test_fused_golden_learning_case(cuda):
    """A reference golden configuration (forcing source, per-row t) with a corrector in the loop."""
    from inc_b200.fused import burgers_cnn_rollout
    from inc_b200.solvers import BurgersSolverTorch
    p, u0, t0, _, scheme = burgers_case(BZ, "rk3_learning_s")
    B, N = u0.shape
    net = _net(4)
    steps = 8
    t_start = np.asarray(t0, dtype=np.float64).reshape(B, 1) if np.ndim(t0) else float(t0)
    ref_f, ref_c = _fp64_loop(net, p, u0, steps, "ssprk3", t0=t_start)
    solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
    solver.t = torch.tensor(t_start, dtype=torch.float32, device=cuda) if np.ndim(t0) else float(t0)
    with torch.no_grad():
        frames, corr = burgers_cnn_rollout(net.float().to(cuda), solver,
                                           torch.tensor(u0, dtype=torch.float32, device=cuda), steps)
    assert rel_l2(frames.cpu().numpy(), ref_f) < TOL
    assert rel_l2(corr.cpu().numpy(), ref_c) < TOL


def test_fused_rejects_unsupported(cuda):
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.fused import burgers_cnn_rollout, cnn_supported
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch
    p = _params(32)
    solver = BurgersSolverTorch(_sim_params(p, 2, "euler", cuda))
    u = torch.zeros(2, 32, device=cuda)
    net = PeriodicCNN1D().to(cuda)
    assert not cnn_supported(net, solver, u)
    with pytest.raises(ValueError):
        burgers_cnn_rollout(net, solver, u, 4)
    p512 = _params(512)
    s512 = BurgersSolverTorch(_sim_params(p512, 2, "euler", cuda))
    u512 = torch.tensor(_u0(2, 512, 2), dtype=torch.float32, device=cuda, requires_grad=True)
    with pytest.raises(ValueError):  # at n = 512 a segment of 27 states does not fit in shared memory
        burgers_cnn_rollout(net, s512, u512, 30, ckpt_every=27)
    small = PeriodicCNN1D(channels=16).to(cuda)
    p = _params(64)
    solver = BurgersSolverTorch(_sim_params(p, 2, "euler", cuda))
    u = torch.tensor(_u0(2, 64, 1), dtype=torch.float32, device=cuda)
    assert not cnn_supported(small, solver, u)
    with torch.no_grad():
        f, c = simulate_rollout(small, solver, u, 3, "INC")  # falls back to the per-step loop
    assert f.shape == (2, 3, 64) and c.shape == (2, 3, 64)


@pytest.mark.parametrize("N,B", [(256, 7), (64, 7)])
def test_fused_training_gradients_are_deterministic(cuda, N, B):
    """Two runs of the fused backward give bit-identical gradients: every weight-gradient
    sum (across the steps and warps of a CTA, then across CTAs) is taken in a fixed order."""
    from inc_b200.fused import burgers_cnn_rollout
    from inc_b200.solvers import BurgersSolverTorch
    steps = 9
    p = _params(N, B=B, seed=11)
    u0_np = _u0(B, N, seed=12)

    def run():
        net = _net(5).float().to(cuda)
        solver = BurgersSolverTorch(_sim_params(p, B, "ssprk3", cuda))
        u0 = torch.tensor(u0_np, dtype=torch.float32, device=cuda, requires_grad=True)
        f, c = burgers_cnn_rollout(net, solver, u0, steps, ckpt_every=4)
        (f.square().sum() + c.square().sum()).backward()
        return [u0.grad.clone()] + [q.grad.clone() for q in net.parameters()]

    a, b = run(), run()
    for x, y in zip(a, b):
        assert torch.equal(x, y)
