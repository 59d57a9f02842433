"""Empty batches (zero trajectories) through the drop-in classes (GPU).

The reference's solvers are torch expressions, so a [0, N] state goes through
them and comes back as a [0, N] tensor; simulate_rollout returns [0, mstep, N]
frames.  The same calls here return the same shapes without a kernel launch,
and the library keeps working for the next, non-empty batch."""
from types import SimpleNamespace

import pytest
import torch

pytestmark = pytest.mark.gpu


def _burgers(cuda, N=256, scheme="ssprk3"):
    from inc_b200.solvers import BurgersSolverTorch
    return BurgersSolverTorch(SimpleNamespace(resolution=N, dt=0.01, x=None, adaptive_CFL=None, L=6.283185307179586,
                                              nu=0.01, device=cuda, convection_term="WENO",
                                              equation_type="viscosity", batch_size=0, time_scheme=scheme))


def _ks(cuda, N=256):
    from inc_b200.solvers import KSSolverTorch
    return KSSolverTorch(SimpleNamespace(resolution=N, dt=0.25, device=cuda, domain_size=torch.zeros(0, device=cuda),
                                         alpha=torch.zeros(0, device=cuda), time_scheme="ETRK2"))


@pytest.mark.parametrize("scheme", ["euler", "ssprk3"])
def test_burgers_step_and_rollout_empty(cuda, scheme):
    from inc_b200.rollout import burgers_rollout
    solver = _burgers(cuda, scheme=scheme)
    u = torch.zeros(0, 256, device=cuda, requires_grad=True)
    out = solver.step(u)
    assert out.shape == (0, 256) and abs(solver.t - 0.01) < 1e-12
    frames = burgers_rollout(solver, u, 5)
    assert frames.shape == (0, 5, 256)
    frames.sum().backward()
    assert u.grad.shape == (0, 256)


def test_ks_step_and_rollout_empty(cuda):
    from inc_b200.rollout import ks_rollout
    solver = _ks(cuda)
    u = torch.zeros(0, 256, device=cuda, requires_grad=True)
    L = torch.zeros(0, device=cuda)
    assert solver.step(u, L).shape == (0, 256)
    frames = ks_rollout(solver, u, 4, L)
    assert frames.shape == (0, 4, 256)
    frames.sum().backward()
    assert u.grad.shape == (0, 256)


def test_simulate_rollout_empty_with_correctors(cuda):
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.rollout import simulate_rollout
    cnn = PeriodicCNN1D().to(cuda)
    u = torch.zeros(0, 256, device=cuda, requires_grad=True)
    res, cor = simulate_rollout(cnn, _burgers(cuda), u, 3, "INC", checkpoint_every=2)
    assert res.shape == (0, 3, 256) and cor.shape == (0, 3, 256)
    with torch.no_grad():
        res, _ = simulate_rollout(cnn, _burgers(cuda), u, 3, "INC")
    assert res.shape == (0, 3, 256)
    # (an FNO corrector is left out: torch's cuFFT rejects a batch of zero
    # transforms, in the reference's FNO as in this one)
    L = torch.zeros(0, device=cuda)
    res, cor = simulate_rollout(None, _ks(cuda), u, 2, None, L=L)
    assert res.shape == (0, 2, 256) and cor is None


def test_weno_reconstruction_empty_then_nonempty(cuda):
    from inc_b200.ops import weno_reconstruction
    assert weno_reconstruction(torch.zeros(0, 64, device=cuda)).shape == (0, 64)
    # the next, non-empty call runs normally
    f = torch.randn(3, 64, device=cuda)
    out = weno_reconstruction(f)
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
