"""CUDA-graph replay of corrector-in-the-loop rollouts (GPU): the replayed graph
gives the same frames and corrections as the eager loop, for new initial states."""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _eager(model, solver, u0, steps, L=None):
    u, fr, cr = u0, [], []
    with torch.no_grad():
        for _ in range(steps):
            s = model(u) if L is None else model(u, L)
            solver.correction_s = s
            u = solver.step(u) if L is None else solver.step(u, L)
            fr.append(u)
            cr.append(s)
    return torch.stack(fr, 1), torch.stack(cr, 1)


def test_graphed_ks_fno_matches_eager(cuda):
    from inc_b200.correctors import FNO1D
    from inc_b200.graphs import GraphedRollout
    from inc_b200.solvers import KSSolverTorch
    torch.manual_seed(0)
    B, N, steps = 6, 64, 5
    L = torch.tensor([22.0, 30.0, 22.0, 40.0, 35.0, 22.0], device=cuda)

    def solver():
        return KSSolverTorch(SimpleNamespace(resolution=N, dt=0.05, device=cuda, domain_size=L,
                                             alpha=torch.zeros(B, device=cuda), time_scheme="ETRK2"))
    net = FNO1D(L=16, modes=4, width=8).to(cuda)
    g = torch.Generator().manual_seed(1)
    u_a = torch.randn(B, N, generator=g).to(cuda)
    u_b = torch.randn(B, N, generator=g).to(cuda)
    gr = GraphedRollout(net, solver(), u_a, steps, domain_size=L)
    for u0 in (u_a, u_b, u_a):
        f, c = gr(u0)
        fe, ce = _eager(net, solver(), u0, steps, L)
        assert torch.allclose(f, fe, rtol=1e-6, atol=1e-6)
        assert torch.allclose(c, ce, rtol=1e-6, atol=1e-6)


def test_graphed_burgers_forcing_matches_eager(cuda):
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.graphs import GraphedRollout
    from inc_b200.solvers import BurgersSolverTorch
    torch.manual_seed(2)
    B, N, steps, J = 5, 128, 6, 3
    rng = np.random.default_rng(3)
    f = lambda a: torch.tensor(a, dtype=torch.float32, device=cuda)  # noqa: E731

    def solver():
        sp = SimpleNamespace(resolution=N, dt=0.004, x=f(np.arange(N) * 2 * math.pi / N), adaptive_CFL=None,
                             L=2 * math.pi, nu=0.01, device=cuda, convection_term="WENO",
                             equation_type="learning", batch_size=B, J=J,
                             A=f(np.full((B, 1, J), 0.3)), omega=f(np.full((B, 1, J), 0.7)),
                             phi=f(np.zeros((B, 1, J))), l=f(np.ones((B, 1, J))), time_scheme="ssprk3")
        s = BurgersSolverTorch(sp)
        s.t = 0.25
        return s
    net = PeriodicCNN1D(channels=16).to(cuda)  # not the fused kernel's shape: the per-step loop is recorded
    u_a = f(rng.uniform(-0.5, 0.5, (B, N)))
    u_b = f(rng.uniform(-0.5, 0.5, (B, N)))
    s_g = solver()
    gr = GraphedRollout(net, s_g, u_a, steps)
    for u0 in (u_b, u_a):
        fr, cr = gr(u0)
        fe, ce = _eager(net, solver(), u0, steps)
        assert torch.allclose(fr, fe, rtol=1e-6, atol=1e-6)
        assert torch.allclose(cr, ce, rtol=1e-6, atol=1e-6)
        assert abs(float(s_g.t) - (0.25 + steps * 0.004)) < 1e-9


def test_graphed_rejects_adaptive_and_shape(cuda):
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.graphs import GraphedRollout
    from inc_b200.solvers import BurgersSolverTorch
    sp = SimpleNamespace(resolution=64, dt=0.01, x=None, adaptive_CFL=0.5, L=2 * math.pi, nu=0.01, device=cuda,
                         convection_term="WENO", equation_type="viscosity", batch_size=2)
    net = PeriodicCNN1D(channels=8).to(cuda)
    u = torch.zeros(2, 64, device=cuda)
    with pytest.raises(ValueError):
        GraphedRollout(net, BurgersSolverTorch(sp), u, 3)
    sp.adaptive_CFL = None
    gr = GraphedRollout(net, BurgersSolverTorch(sp), u, 3)
    with pytest.raises(ValueError):
        gr(torch.zeros(3, 64, device=cuda))


@pytest.mark.parametrize("B,n", [(8, 128), (40, 256)])
def test_graphed_burgers_rollout_backward_matches_eager(cuda, B, n):
    """A differentiable rollout (forward + checkpointed backward: at these batches the
    adjoint runs on a cluster of three or two CTAs per row) captured in one CUDA graph
    and replayed for new inputs gives the eager gradients."""
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    L, steps = 2 * math.pi, 20
    sp = SimpleNamespace(resolution=n, dt=0.2 / n, x=None, adaptive_CFL=None, L=L, nu=0.01, device=cuda,
                         convection_term="WENO", equation_type="viscosity", batch_size=B, time_scheme="ssprk3",
                         cells_per_thread=1)
    x = torch.arange(n, device=cuda) * (L / n)
    g = torch.Generator().manual_seed(n + B)
    amp = lambda: (torch.rand(B, 1, generator=g) - 0.5).to(cuda)  # noqa: E731
    w = torch.randn(B, steps, n, generator=g).to(cuda)

    def grads(u_in, solver):
        u = u_in.clone().requires_grad_(True)
        fr = burgers_rollout(solver, u, steps, ckpt_every=8)
        (gu,) = torch.autograd.grad((fr * w).sum(), (u,))
        return gu

    u_a = amp() * torch.sin(x) + amp() * torch.cos(2 * x)
    u_b = amp() * torch.sin(3 * x) + amp() * torch.cos(x)
    static_u = u_a.clone()
    solver = BurgersSolverTorch(sp)
    side = torch.cuda.Stream(cuda)
    side.wait_stream(torch.cuda.current_stream(cuda))
    with torch.cuda.stream(side):
        for _ in range(2):
            grads(static_u, solver)
    torch.cuda.current_stream(cuda).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        static_g = grads(static_u, solver)
    for u_in in (u_a, u_b):
        static_u.copy_(u_in)
        graph.replay()
        torch.cuda.synchronize()
        ref = grads(u_in, BurgersSolverTorch(sp))
        assert torch.isfinite(static_g).all()
        assert torch.equal(static_g, ref)
