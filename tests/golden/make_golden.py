"""Generate golden vectors by running the reference's own 1D solvers in FP64.

Run from the repository root with the path of a checkout of the reference
(``--reference PATH``, or the ``INC_REFERENCE`` environment variable; there is
no default):

    python tests/golden/make_golden.py --reference PATH

It imports ``solvers/solver_1d.py`` from the reference (never copied), runs it
with ``torch.set_default_dtype(torch.float64)`` on seeded inputs, and writes
``tests/golden/*.npz``.  The files are small and committed: the GPU test box
has no reference tree.

The only change to the reference's behaviour is the Burgers ``step`` arity
fix: the shipped ``step`` calls ``u, source = self._apply_corrections(u, source)``
(solver_1d.py:188) against a one-argument ``_apply_corrections`` (solver_1d.py:116)
and raises ``TypeError``.  ``_FixedBurgers`` below builds the step from the
reference's own methods with ``source = self._apply_corrections(source)``.
SSP-RK3 is composed from the same methods (the reference only has Euler).
"""
from __future__ import annotations

import math
import os
import sys
from types import SimpleNamespace

import numpy as np
import torch

REF = None  # the reference checkout, set by main()
OUT = os.path.dirname(os.path.abspath(__file__))
BurgersSolverTorch = KSSolverTorch = weno_reconstruction = _FixedBurgers = None


def _import_reference(ref):
    """Import the reference's solvers/solver_1d.py from the checkout at `ref` and
    bind the module-level names the generators use."""
    global REF, BurgersSolverTorch, KSSolverTorch, weno_reconstruction, _FixedBurgers
    REF = os.path.abspath(ref)
    if not os.path.isfile(os.path.join(REF, "solvers", "solver_1d.py")):
        raise SystemExit(f"{REF} is not a checkout of the reference (no solvers/solver_1d.py)")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    from solvers.solver_1d import BurgersSolverTorch, KSSolverTorch, weno_reconstruction
    _FixedBurgers = _fixed_burgers(BurgersSolverTorch)


def _fixed_burgers(base):
    class _FixedBurgers(base):
        """Reference solver with the ``_apply_corrections`` call fixed."""

        def rhs_at(self, u, t):
            saved = self.t
            self.t = t
            source = self._compute_source(u)
            self.t = saved
            source = self._apply_corrections(source)
            return self.calc_nonlinear(u) + self.calc_linear(u) + source

        def step(self, u):
            if self.adaptive_CFL is not None:
                return self.step_adaptive(u)
            u_new = u + self.dt * self.rhs_at(u, self.t)
            self.t += self.dt
            return u_new

        def step_rk3(self, u):
            dt, t = self.dt, self.t
            u1 = u + dt * self.rhs_at(u, t)
            u2 = 0.75 * u + 0.25 * (u1 + dt * self.rhs_at(u1, t + dt))
            u3 = (1.0 / 3.0) * u + (2.0 / 3.0) * (u2 + dt * self.rhs_at(u2, t + 0.5 * dt))
            self.t = t + dt
            return u3

        def step_adaptive(self, u):
            target, substeps = self.dt, 0
            while target > 0:
                max_u = torch.max(torch.abs(u))
                allowed = self.adaptive_CFL * self.dx / max_u.item() if max_u.item() > 0 else target
                dt_local = min(target, allowed)
                u = u + dt_local * self.rhs_at(u, self.t)
                self.t += dt_local
                target -= dt_local
                if int(math.ceil(target / dt_local)) > 1000:
                    break
                substeps += 1
            self.substeps = substeps
            return u

    return _FixedBurgers


def burgers_params(rng, B, N, *, eq="viscosity", conv="WENO", nu_rows=False, J=3,
                   adaptive=None, dt=0.01, L=2 * math.pi):
    x = torch.arange(N, dtype=torch.float64) * (L / N)
    p = SimpleNamespace(resolution=N, dt=dt, x=x, adaptive_CFL=adaptive, L=L,
                        nu=(torch.from_numpy(rng.uniform(0.005, 0.05, (B, 1))) if nu_rows else 0.01),
                        device="cpu", convection_term=conv, equation_type=eq, batch_size=B,
                        beta=torch.from_numpy(rng.uniform(-0.5, 0.5, (B, 1))), J=J,
                        A=torch.from_numpy(rng.uniform(-0.5, 0.5, (B, 1, J))),
                        omega=torch.from_numpy(rng.uniform(-0.4, 0.4, (B, 1, J))),
                        phi=torch.from_numpy(rng.uniform(0, 2 * math.pi, (B, 1, J))),
                        l=torch.from_numpy(rng.integers(1, 4, (B, 1, J)).astype(np.float64)))
    return p


def sines_u0(rng, B, N, K=5, L=2 * math.pi):
    x = np.arange(N) * (L / N)
    a = rng.uniform(-0.5, 0.5, (B, K))
    ph = rng.uniform(0, 2 * math.pi, (B, K))
    k = np.arange(1, K + 1)
    return (a[:, :, None] * np.sin(k[None, :, None] * x[None, None, :] * (2 * math.pi / L)
                                   + ph[:, :, None])).sum(1)


def p_to_dict(prefix, p):
    d = {f"{prefix}N": p.resolution, f"{prefix}dt": p.dt, f"{prefix}L": p.L,
         f"{prefix}x": p.x.numpy(), f"{prefix}conv": p.convection_term,
         f"{prefix}eq": p.equation_type,
         f"{prefix}nu": (p.nu.numpy() if torch.is_tensor(p.nu) else np.float64(p.nu)),
         f"{prefix}beta": p.beta.numpy(), f"{prefix}A": p.A.numpy(),
         f"{prefix}omega": p.omega.numpy(), f"{prefix}phi": p.phi.numpy(),
         f"{prefix}l": p.l.numpy(),
         f"{prefix}cfl": (np.float64(p.adaptive_CFL) if p.adaptive_CFL is not None else np.float64(np.nan))}
    return d


def make_burgers():
    rng = np.random.default_rng(1234)
    out = {}
    # Per-op: WENO reconstruction both directions, nonlinear and linear terms.
    f = rng.standard_normal((3, 16))
    out["weno_f"] = f
    out["weno_left"] = weno_reconstruction(torch.from_numpy(f), "left").numpy()
    out["weno_right"] = weno_reconstruction(torch.from_numpy(f), "right").numpy()
    p = burgers_params(rng, 3, 32)
    solver = _FixedBurgers(p)
    u = torch.from_numpy(sines_u0(rng, 3, 32))
    out["op_u"] = u.numpy()
    out["op_nonlinear_weno"] = solver.calc_nonlinear_weno(u).numpy()
    out["op_linear"] = solver.calc_linear(u).numpy()

    cases = [
        ("euler_visc", dict(eq="viscosity"), "euler", False),
        ("euler_learning", dict(eq="learning", nu_rows=True), "euler", True),
        ("euler_linear_fdm", dict(eq="linear", conv="FDM"), "euler", True),
        ("rk3_visc", dict(eq="viscosity"), "rk3", False),
        ("rk3_learning_s", dict(eq="learning", nu_rows=True), "rk3", True),
        ("rk3_linear", dict(eq="linear"), "rk3", True),
        ("adaptive_visc", dict(eq="viscosity", adaptive=0.2, dt=0.05), "euler", False),
    ]
    names = []
    for name, kw, scheme, with_s in cases:
        B, N, steps = 4, 64, 5
        p = burgers_params(rng, B, N, **kw)
        u0 = sines_u0(rng, B, N)
        s = 0.1 * rng.standard_normal((B, N)) if with_s else None
        t0 = rng.uniform(0, 1, (B, 1))
        solver = _FixedBurgers(p)
        solver.t = torch.from_numpy(t0.copy())
        solver.correction_s = torch.from_numpy(s) if s is not None else None
        u = torch.from_numpy(u0)
        frames = []
        for _ in range(steps):
            u = solver.step_rk3(u) if scheme == "rk3" else solver.step(u)
            frames.append(u.numpy().copy())
        out.update(p_to_dict(f"{name}.", p))
        out[f"{name}.scheme"] = scheme
        out[f"{name}.u0"] = u0
        out[f"{name}.t0"] = t0
        out[f"{name}.s"] = s if s is not None else np.zeros(0)
        out[f"{name}.frames"] = np.stack(frames, 1)
        if kw.get("adaptive") is not None:
            out[f"{name}.substeps"] = np.int64(solver.substeps)
        names.append(name)
    out["cases"] = np.array(names)

    # Gradients by torch autograd through the (fixed) reference, one and three steps.
    gnames = []
    for name, scheme, eq, steps in [("g_euler", "euler", "learning", 1), ("g_rk3", "rk3", "linear", 1),
                                    ("g_rk3_3", "rk3", "viscosity", 3), ("g_euler_fdm3", "euler", "linear", 3)]:
        B, N = 3, 32
        p = burgers_params(rng, B, N, eq=eq, conv=("FDM" if "fdm" in name else "WENO"), nu_rows=True)
        u0 = torch.from_numpy(sines_u0(rng, B, N)).requires_grad_(True)
        s = torch.from_numpy(0.1 * rng.standard_normal((B, N))).requires_grad_(True)
        w = torch.from_numpy(rng.standard_normal((B, steps, N)))
        solver = _FixedBurgers(p)
        solver.t = torch.from_numpy(rng.uniform(0, 1, (B, 1)))
        t0 = solver.t.numpy().copy()
        solver.correction_s = s
        u, frames = u0, []
        for _ in range(steps):
            u = solver.step_rk3(u) if scheme == "rk3" else solver.step(u)
            frames.append(u)
        loss = (torch.stack(frames, 1) * w).sum()
        gu, gs = torch.autograd.grad(loss, (u0, s))
        out.update(p_to_dict(f"{name}.", p))
        out[f"{name}.scheme"] = scheme
        out[f"{name}.steps"] = np.int64(steps)
        out[f"{name}.u0"] = u0.detach().numpy()
        out[f"{name}.t0"] = t0
        out[f"{name}.s"] = s.detach().numpy()
        out[f"{name}.w"] = w.numpy()
        out[f"{name}.loss"] = np.float64(loss.item())
        out[f"{name}.grad_u"] = gu.numpy()
        out[f"{name}.grad_s"] = gs.numpy()
        gnames.append(name)
    out["grad_cases"] = np.array(gnames)
    np.savez_compressed(os.path.join(OUT, "burgers_golden.npz"), **out)


def ks_u0(rng, B, N, L):
    x = np.arange(N) * (L / N)
    k = np.arange(1, 9)
    a = rng.standard_normal((B, 8)) / k
    ph = rng.uniform(0, 2 * math.pi, (B, 8))
    return (a[:, :, None] * np.cos(2 * math.pi * k[None, :, None] * x[None, None, :] / L
                                   + ph[:, :, None])).sum(1)


def make_ks():
    rng = np.random.default_rng(4321)
    out = {}
    names = []
    cases = [
        ("etrk2_same_L", "ETRK2", 64, [64.0] * 4, 0.25, True, False, 4),
        ("etrk2_ragged_L", "ETRK2", 64, [48.0, 64.0, 80.0, 100.0, 22.0], 0.1, True, True, 3),
        ("etd1_small_dt", "ETD1", 32, [32.0, 40.0, 50.0], 0.05, True, True, 3),
        ("etrk2_n128_nos", "ETRK2", 128, [100.0, 100.0], 0.2, False, False, 3),
    ]
    for name, scheme, N, Ls, dt, with_s, with_cu, steps in cases:
        B = len(Ls)
        ds = torch.tensor(Ls)
        sp = SimpleNamespace(resolution=N, dt=dt, device="cpu", domain_size=ds,
                             alpha=torch.zeros(B), time_scheme=scheme)
        solver = KSSolverTorch(sp)
        u0 = np.stack([ks_u0(rng, 1, N, L)[0] for L in Ls])
        s = 0.01 * rng.standard_normal((B, N)) if with_s else None
        cu = 0.01 * rng.standard_normal((B, N)) if with_cu else None
        solver.correction_s = torch.from_numpy(s) if s is not None else None
        solver.correction_u = torch.from_numpy(cu) if cu is not None else None
        u = torch.from_numpy(u0)
        frames = []
        for _ in range(steps):
            u = solver.step(u, ds)
            frames.append(u.numpy().copy())
        out[f"{name}.scheme"] = scheme
        out[f"{name}.N"] = np.int64(N)
        out[f"{name}.L"] = np.array(Ls)
        out[f"{name}.dt"] = np.float64(dt)
        out[f"{name}.u0"] = u0
        out[f"{name}.s"] = s if s is not None else np.zeros(0)
        out[f"{name}.cu"] = cu if cu is not None else np.zeros(0)
        out[f"{name}.frames"] = np.stack(frames, 1)
        # single substeps, straight from the reference's etd1_step / etrk2_step
        sub = solver.etrk2_step if scheme == "ETRK2" else solver.etd1_step
        out[f"{name}.substep"] = sub(torch.from_numpy(u0), ds).numpy()
        names.append(name)
    out["cases"] = np.array(names)

    gnames = []
    for name, scheme, N, Ls, dt, steps in [("g_etrk2", "ETRK2", 64, [64.0, 64.0, 50.0], 0.25, 1),
                                           ("g_etrk2_3", "ETRK2", 32, [40.0, 40.0], 0.2, 3),
                                           ("g_etd1", "ETD1", 32, [30.0, 36.0], 0.05, 2)]:
        B = len(Ls)
        ds = torch.tensor(Ls)
        sp = SimpleNamespace(resolution=N, dt=dt, device="cpu", domain_size=ds,
                             alpha=torch.zeros(B), time_scheme=scheme)
        solver = KSSolverTorch(sp)
        u0 = torch.from_numpy(np.stack([ks_u0(rng, 1, N, L)[0] for L in Ls])).requires_grad_(True)
        s = torch.from_numpy(0.01 * rng.standard_normal((B, N))).requires_grad_(True)
        w = torch.from_numpy(rng.standard_normal((B, steps, N)))
        solver.correction_s = s
        u, frames = u0, []
        for _ in range(steps):
            u = solver.step(u, ds)
            frames.append(u)
        loss = (torch.stack(frames, 1) * w).sum()
        gu, gs = torch.autograd.grad(loss, (u0, s))
        out[f"{name}.scheme"] = scheme
        out[f"{name}.N"] = np.int64(N)
        out[f"{name}.L"] = np.array(Ls)
        out[f"{name}.dt"] = np.float64(dt)
        out[f"{name}.steps"] = np.int64(steps)
        out[f"{name}.u0"] = u0.detach().numpy()
        out[f"{name}.s"] = s.detach().numpy()
        out[f"{name}.w"] = w.numpy()
        out[f"{name}.loss"] = np.float64(loss.item())
        out[f"{name}.grad_u"] = gu.numpy()
        out[f"{name}.grad_s"] = gs.numpy()
        gnames.append(name)
    out["grad_cases"] = np.array(gnames)
    np.savez_compressed(os.path.join(OUT, "ks_golden.npz"), **out)


def _reference_fno_module():
    """models/models_1d/fno.py imported by file path.  Its package __init__ imports
    modules the reference does not ship, so a bare package object stands in for
    ``models.models_1d``; fno.py's ``from .utils import get_grid`` then loads the
    reference's utils.py from the same directory."""
    import importlib.util
    import types
    name = "_ref_models_1d"
    if name not in sys.modules:
        pkg = types.ModuleType(name)
        pkg.__path__ = [os.path.join(REF, "models", "models_1d")]
        sys.modules[name] = pkg
    if f"{name}.fno" not in sys.modules:
        spec = importlib.util.spec_from_file_location(f"{name}.fno", os.path.join(REF, "models", "models_1d", "fno.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"{name}.fno"] = m
        spec.loader.exec_module(m)
    return sys.modules[f"{name}.fno"]


def _fno64(cls, **kw):
    """A reference FNO1D initialised as a float32 model (the RNG stream of its default
    construction), then run in FP64: real parameters to float64, the complex64
    weights1 to complex128 (same values)."""
    prev = torch.get_default_dtype()
    torch.set_default_dtype(torch.float32)
    try:
        net = cls(**kw)
    finally:
        torch.set_default_dtype(prev)
    for m in net.modules():
        for pn, prm in list(m.named_parameters(recurse=False)):
            dt = torch.complex128 if prm.is_complex() else torch.float64
            setattr(m, pn, torch.nn.Parameter(prm.detach().to(dt)))
    return net


def make_fno():
    """The reference's FNO corrector (models/models_1d/fno.py:39-105) in FP64: outputs for
    the three grid forms of get_grid (L=None -> self.L, a float, a per-row tensor) and
    gradients of a weighted sum w.r.t. the input and every parameter.  Small case: all
    parameters and gradients stored.  Benchmark-sized case (width 64, 16 modes): the
    network is rebuilt from its seed, so only parameter checksums, outputs, the input
    gradient and each parameter gradient's projection on a seeded direction are stored."""
    FNO1D = _reference_fno_module().FNO1D
    rng = np.random.default_rng(55)
    out = {}
    for name, seed, kw, (B, N) in (("f_small", 21, dict(L=16, modes=4, width=8), (3, 32)),
                                   ("f_bench", 22, dict(L=16, modes=16, width=64), (2, 128))):
        torch.manual_seed(seed)
        net = _fno64(FNO1D, **kw)
        x = torch.from_numpy(rng.standard_normal((B, N)))
        Lt = torch.from_numpy(rng.uniform(20, 60, B))
        out[f"{name}.seed"] = np.int64(seed)
        out[f"{name}.kw"] = np.array([kw["L"], kw["modes"], kw["width"]], dtype=np.int64)
        out[f"{name}.x"] = x.numpy()
        out[f"{name}.Lt"] = Lt.numpy()
        with torch.no_grad():
            out[f"{name}.y_none"] = net(x).numpy()
            out[f"{name}.y_float"] = net(x, 5.0).numpy()
        xg = x.clone().requires_grad_(True)
        y = net(xg, Lt)
        w = torch.from_numpy(rng.standard_normal((B, N)))
        grads = torch.autograd.grad((y * w).sum(), [xg] + list(net.parameters()))
        out[f"{name}.y_tensor"] = y.detach().numpy()
        out[f"{name}.w"] = w.numpy()
        out[f"{name}.grad_x"] = grads[0].numpy()
        g = torch.Generator().manual_seed(seed)
        for (pn, prm), gp in zip(net.named_parameters(), grads[1:]):
            d = torch.randn(prm.shape, generator=g, dtype=torch.float64)
            gr = torch.view_as_real(gp).double() if gp.is_complex() else gp.double()
            pr = torch.view_as_real(prm.detach()).double() if prm.is_complex() else prm.detach().double()
            if gp.is_complex():
                d = torch.stack([d, torch.randn(prm.shape, generator=g, dtype=torch.float64)], -1)
            out[f"{name}.pgrad_proj.{pn}"] = np.float64((gr * d).sum())
            out[f"{name}.param_sum.{pn}"] = np.float64(pr.sum())
            if name == "f_small":
                out[f"{name}.param.{pn}"] = pr.numpy()
                out[f"{name}.pgrad.{pn}"] = gr.numpy()
    np.savez_compressed(os.path.join(OUT, "fno_golden.npz"), **out)


def make_hybrid():
    """A corrector network in the loop: s = net(u) before every reference step()
    (trainer_1d.py:168-175), loss = MSE(frames, target), FP64 autograd."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(OUT)))
    from inc_b200.correctors import PeriodicCNN1D
    FNO1D = _reference_fno_module().FNO1D
    rng = np.random.default_rng(77)
    out = {}
    # Burgers, SSP-RK3 and Euler, with a periodic CNN corrector
    for name, scheme in (("h_burgers_rk3", "rk3"), ("h_burgers_euler", "euler")):
        torch.manual_seed(5)
        B, N, steps = 3, 32, 3
        net = PeriodicCNN1D(channels=4, kernel=5, layers=4)
        p = burgers_params(rng, B, N, eq="viscosity", nu_rows=False)
        solver = _FixedBurgers(p)
        u0 = torch.from_numpy(sines_u0(rng, B, N)).requires_grad_(True)
        target = torch.from_numpy(rng.standard_normal((B, steps, N)) * 0.3)
        u, frames = u0, []
        for _ in range(steps):
            solver.correction_s = net(u)
            u = solver.step_rk3(u) if scheme == "rk3" else solver.step(u)
            frames.append(u)
        loss = torch.mean((torch.stack(frames, 1) - target) ** 2)
        params = list(net.parameters())
        grads = torch.autograd.grad(loss, [u0] + params)
        out.update(p_to_dict(f"{name}.", p))
        out[f"{name}.scheme"] = scheme
        out[f"{name}.u0"] = u0.detach().numpy()
        out[f"{name}.target"] = target.numpy()
        out[f"{name}.loss"] = np.float64(loss.item())
        out[f"{name}.grad_u"] = grads[0].numpy()
        for (pn, prm), g in zip(net.named_parameters(), grads[1:]):
            out[f"{name}.param.{pn}"] = prm.detach().numpy()
            out[f"{name}.pgrad.{pn}"] = g.numpy()
    # KS ETRK2 with an FNO corrector taking the domain size
    torch.manual_seed(6)
    name = "h_ks"
    B, N, steps, dt = 2, 32, 2, 0.2
    Ls = [32.0, 40.0]
    net = _fno64(FNO1D, L=16, modes=4, width=8)  # the reference's own FNO corrector
    ds = torch.tensor(Ls)
    sp = SimpleNamespace(resolution=N, dt=dt, device="cpu", domain_size=ds, alpha=torch.zeros(B),
                         time_scheme="ETRK2")
    solver = KSSolverTorch(sp)
    u0 = torch.from_numpy(np.stack([ks_u0(rng, 1, N, L)[0] for L in Ls])).requires_grad_(True)
    target = torch.from_numpy(rng.standard_normal((B, steps, N)) * 0.3)
    u, frames = u0, []
    for _ in range(steps):
        solver.correction_s = net(u, ds)
        u = solver.step(u, ds)
        frames.append(u)
    loss = torch.mean((torch.stack(frames, 1) - target) ** 2)
    grads = torch.autograd.grad(loss, [u0] + list(net.parameters()))
    out[f"{name}.N"] = np.int64(N)
    out[f"{name}.L"] = np.array(Ls)
    out[f"{name}.dt"] = np.float64(dt)
    out[f"{name}.u0"] = u0.detach().numpy()
    out[f"{name}.target"] = target.numpy()
    out[f"{name}.loss"] = np.float64(loss.item())
    out[f"{name}.grad_u"] = grads[0].numpy()
    for (pn, prm), g in zip(net.named_parameters(), grads[1:]):
        out[f"{name}.param.{pn}"] = prm.detach().numpy()
        out[f"{name}.pgrad.{pn}"] = g.numpy()
    np.savez_compressed(os.path.join(OUT, "hybrid_golden.npz"), **out)


def _load_reference_module(relpath, name):
    """Import one reference file; plotting libraries absent here are stubbed
    (the functions used below only call numpy and torch)."""
    import importlib.util
    import types
    from unittest import mock
    for mod in ("matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(mod, mock.MagicMock(name=mod))
    spec = importlib.util.spec_from_file_location(name, os.path.join(REF, relpath))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def make_analysis_and_data():
    """Energy spectrum (analysis/Plot_KS.py:196-235) and trajectory windows
    (data/data_loader_1d.py:8-139) from the reference's own code."""
    rng = np.random.default_rng(99)
    out = {}
    pks = _load_reference_module("analysis/Plot_KS.py", "ref_plot_ks")
    for name, shape in (("spec_even", (3, 4, 64)), ("spec_even2d", (5, 32)), ("spec_256", (2, 3, 256))):
        v = rng.standard_normal(shape).astype(np.float32)
        e, k = pks.calculate_energy_spectrum(v)
        out[f"{name}.v"] = v
        out[f"{name}.energy"] = e.numpy().astype(np.float64)
        out[f"{name}.k"] = k.numpy().astype(np.float64)
    dl = _load_reference_module("data/data_loader_1d.py", "ref_data_loader")
    B, T1, D, J = 3, 13, 16, 2
    data = {"trajectories": torch.from_numpy(rng.standard_normal((B, T1, D))),
            "nu": torch.from_numpy(rng.uniform(0.01, 0.05, (B, 1))),
            "A": torch.from_numpy(rng.standard_normal((B, 1, J))), "omega": torch.from_numpy(rng.standard_normal((B, 1, J))),
            "phi": torch.from_numpy(rng.standard_normal((B, 1, J))), "l": torch.from_numpy(rng.standard_normal((B, 1, J))),
            "domain_size": torch.from_numpy(rng.uniform(20, 60, (B, 1))),
            "metadata": {"gen_dt": 0.5}}
    out["dl.trajectories"] = data["trajectories"].numpy()
    for k in ("nu", "A", "omega", "phi", "l", "domain_size"):
        out[f"dl.{k}"] = data[k].numpy()
    cases = []
    for cname, cls, dt, mstep, gap in (("bg_r1", dl.BurgersDataset, 0.5, 3, 1), ("bg_r2", dl.BurgersDataset, 1.0, 2, 3),
                                       ("ks_r1", dl.KSDataset, 0.5, 4, 2), ("ks_r3", dl.KSDataset, 1.5, 2, 3)):
        ds = cls(data, dt=dt, mstep=mstep, starts_gap=gap)
        items = [ds[i] for i in range(len(ds))]
        out[f"dl.{cname}.args"] = np.array([dt, mstep, -1 if gap is None else gap], dtype=np.float64)
        out[f"dl.{cname}.len"] = np.int64(len(ds))
        out[f"dl.{cname}.u_initial"] = torch.stack([it["u_initial"] for it in items]).numpy()
        out[f"dl.{cname}.u_target"] = torch.stack([it["u_target"] for it in items]).numpy()
        if cls is dl.BurgersDataset:
            out[f"dl.{cname}.t"] = np.array([float(it["t"]) for it in items])
            out[f"dl.{cname}.nu"] = torch.stack([it["nu"] for it in items]).numpy()
        else:
            out[f"dl.{cname}.domain_size"] = torch.stack([it["domain_size"] for it in items]).numpy()
        cases.append(cname)
    out["dl.cases"] = np.array(cases)
    np.savez_compressed(os.path.join(OUT, "analysis_data_golden.npz"), **out)


def main():
    import argparse
    gens = {"burgers": make_burgers, "ks": make_ks, "hybrid": make_hybrid, "analysis_data": make_analysis_and_data,
            "fno": make_fno}
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--reference", default=os.environ.get("INC_REFERENCE"),
                    help="checkout of the reference (default: $INC_REFERENCE; required)")
    ap.add_argument("--only", nargs="+", choices=sorted(gens), default=sorted(gens),
                    help="golden files to (re)generate (default: all)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("the reference checkout is required: --reference PATH or INC_REFERENCE=PATH")
    _import_reference(args.reference)
    torch.set_default_dtype(torch.float64)
    for name in args.only:
        gens[name]()
        f = f"{name}_golden.npz"
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")


if __name__ == "__main__":
    main()
