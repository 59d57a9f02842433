"""Numpy restatement of the reference Burgers solver (test infrastructure only).

Follows ``solvers/solver_1d.py`` of tum-pbs/INC (cited per function).  Arrays are
``[B, N]`` rows of a periodic grid; every function works in the dtype of its
inputs (float64 for the FP64 oracle, float32 for the CPU baseline).

Reference fix applied here (and nowhere else): ``BurgersSolverTorch.step`` calls
``u, source = self._apply_corrections(u, source)`` (solver_1d.py:188 and :166) but
``_apply_corrections(self, source)`` takes one argument and returns one value
(solver_1d.py:116-123), so the shipped ``step`` raises ``TypeError``.  The
intended semantics, used below, are ``source = source + correction_s``.

The reference integrates in time with forward Euler only (solver_1d.py:192).
``step_ssprk3`` composes the reference's own right-hand side (nonlinear + linear
+ source, solver_1d.py:187-191) with the Shu-Osher three-stage SSP-RK3 scheme;
the forcing source is evaluated at the stage times t, t+dt, t+dt/2 and the
correction ``s`` is held constant over the step.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

WENO_EPS = 1e-6          # solver_1d.py:5
WENO_GAMMA = (0.1, 0.6, 0.3)  # solver_1d.py:22 and :33


def roll(f, shift):
    """``torch.roll(f, shifts=shift, dims=-1)``: out[i] = f[i - shift]."""
    return np.roll(f, shift, axis=-1)


def weno_reconstruction(f, direction="left"):
    """WENO5-JS reconstruction with the reference's stencils.

    solver_1d.py:4-42.  'left' reconstructs f+ at interface i+1/2 from
    f[i-2..i+2]; 'right' reconstructs f- from f[i-1..i+3] (the reference's
    right-biased stencils, which land at i+3/2).
    """
    eps = WENO_EPS
    f_m2 = roll(f, 2)
    f_m1 = roll(f, 1)
    f_0 = f
    f_p1 = roll(f, -1)
    f_p2 = roll(f, -2)
    f_p3 = roll(f, -3)
    dt_ = f.dtype.type
    c = lambda v: dt_(v)  # noqa: E731  constants in the working precision
    if direction == "left":                                   # :14-22
        q0 = c(1 / 3) * f_m2 - c(7 / 6) * f_m1 + c(11 / 6) * f_0
        q1 = c(-1 / 6) * f_m1 + c(5 / 6) * f_0 + c(1 / 3) * f_p1
        q2 = c(1 / 3) * f_0 + c(5 / 6) * f_p1 - c(1 / 6) * f_p2
        b0 = c(13 / 12) * (f_m2 - 2 * f_m1 + f_0) ** 2 + c(1 / 4) * (f_m2 - 4 * f_m1 + 3 * f_0) ** 2
        b1 = c(13 / 12) * (f_m1 - 2 * f_0 + f_p1) ** 2 + c(1 / 4) * (f_m1 - f_p1) ** 2
        b2 = c(13 / 12) * (f_0 - 2 * f_p1 + f_p2) ** 2 + c(1 / 4) * (3 * f_0 - 4 * f_p1 + f_p2) ** 2
    elif direction == "right":                                # :24-33
        q0 = c(11 / 6) * f_p1 - c(7 / 6) * f_0 + c(1 / 3) * f_m1
        q1 = c(1 / 3) * f_p2 + c(5 / 6) * f_p1 - c(1 / 6) * f_0
        q2 = -c(1 / 6) * f_p3 + c(5 / 6) * f_p2 + c(1 / 3) * f_p1
        b0 = c(13 / 12) * (f_p1 - 2 * f_0 + f_m1) ** 2 + c(1 / 4) * (3 * f_p1 - 4 * f_0 + f_m1) ** 2
        b1 = c(13 / 12) * (f_p2 - 2 * f_p1 + f_0) ** 2 + c(1 / 4) * (f_p2 - f_0) ** 2
        b2 = c(13 / 12) * (f_p3 - 2 * f_p2 + f_p1) ** 2 + c(1 / 4) * (3 * f_p3 - 4 * f_p2 + f_p1) ** 2
    else:                                                     # :35-36
        raise ValueError("Direction must be 'left' or 'right'.")
    # :39-42  alpha_k = gamma_k / (eps + beta_k)^2, w = alpha / sum(alpha)
    a = [c(g) / (c(eps) + b) ** 2 for g, b in zip(WENO_GAMMA, (b0, b1, b2))]
    s = a[0] + a[1] + a[2]
    return (a[0] / s) * q0 + (a[1] / s) * q1 + (a[2] / s) * q2


def nonlinear_weno(u, dx):
    """-(d/dx) of the Lax-Friedrichs split WENO5 flux; solver_1d.py:129-142.

    alpha is the per-row max |u| (solver_1d.py:133)."""
    h = u.dtype.type(0.5)
    flux = h * u ** 2
    alpha = np.max(np.abs(u), axis=1, keepdims=True)
    fp = h * (flux + alpha * u)
    fm = h * (flux - alpha * u)
    hp = weno_reconstruction(fp, "left")
    hm = weno_reconstruction(fm, "right")
    dp = (hp - roll(hp, 1)) / u.dtype.type(dx)
    dm = (hm - roll(hm, 1)) / u.dtype.type(dx)
    return -(dp + dm)


def nonlinear_fdm(u, dx):
    """-u * D1 u with the periodic central first difference; solver_1d.py:87-93, :125-127."""
    d1 = (roll(u, -1) - roll(u, 1)) * u.dtype.type(1.0 / (2 * dx))
    return -u * d1


def linear(u, nu, dx):
    """nu * D2 u, D2 the periodic central second difference / dx^2.

    solver_1d.py:95-102 and :144-146 (the reference multiplies by the dense
    N x N matrix; its only non-zeros are this three-point stencil)."""
    inv = u.dtype.type(1.0 / dx ** 2)
    return nu * ((roll(u, 1) - 2 * u + roll(u, -1)) * inv)


def forcing(x, t, A, omega, phi, l, L):
    """sum_j A_j sin(omega_j t + 2 pi l_j x / L + phi_j); solver_1d.py:74-85.

    A, omega, phi, l: [B, 1, J]; t: [B, 1] (or scalar); x: [N]."""
    B = A.shape[0]
    x_ = x.reshape(1, -1)
    t = np.full((B, 1), t, dtype=x.dtype) if np.isscalar(t) else np.asarray(t).reshape(B, 1)
    out = np.zeros((B, x.shape[0]), dtype=x.dtype)
    for j in range(A.shape[-1]):
        arg = omega[..., j] * t + (2 * np.pi * l[..., j] / L) * x_ + phi[..., j]
        out += A[..., j] * np.sin(arg)
    return out


@dataclass
class BurgersParams:
    """The sim_params fields the reference Burgers solver reads (solver_1d.py:45-66)."""
    resolution: int
    L: float
    dt: float
    nu: object                      # scalar or [B, 1]
    convection_term: str = "WENO"   # "WENO" | "FDM"
    equation_type: str = "viscosity"  # "homogeneous" | "viscosity" | "linear" | "learning"
    beta: object = 0.0              # scalar or [B, 1] ('linear')
    A: Optional[np.ndarray] = None  # [B, 1, J] ('learning')
    omega: Optional[np.ndarray] = None
    phi: Optional[np.ndarray] = None
    l: Optional[np.ndarray] = None
    x: Optional[np.ndarray] = field(default=None)
    adaptive_CFL: Optional[float] = None

    @property
    def dx(self):
        return self.L / self.resolution   # solver_1d.py:56


def source(u, p: BurgersParams, t):
    """solver_1d.py:104-114."""
    if p.equation_type in ("homogeneous", "viscosity"):
        return u.dtype.type(0.0)
    if p.equation_type == "linear":
        return p.beta * u
    if p.equation_type == "learning":
        return forcing(p.x.astype(u.dtype), t, p.A, p.omega, p.phi, p.l, p.L)
    raise ValueError("Unknown equation type.")


def rhs(u, p: BurgersParams, t, s=None):
    """nonlinear + linear + source (+ correction s); solver_1d.py:187-191."""
    src = source(u, p, t)
    if s is not None:                        # _apply_corrections, :116-123
        src = src + s
    if p.convection_term == "WENO":
        nl = nonlinear_weno(u, p.dx)
    elif p.convection_term == "FDM":
        nl = nonlinear_fdm(u, p.dx)
    else:
        raise ValueError("Convection scheme not recognized")
    return nl + linear(u, p.nu, p.dx) + src


def step_euler(u, p: BurgersParams, t=0.0, s=None, dt=None):
    """Forward Euler step, u + dt * rhs; solver_1d.py:181-195.  Returns (u_new, t + dt)."""
    dt = p.dt if dt is None else dt
    return u + dt * rhs(u, p, t, s), t + dt


def step_ssprk3(u, p: BurgersParams, t=0.0, s=None, dt=None):
    """Shu-Osher SSP-RK3 on the reference right-hand side.  Returns (u_new, t + dt)."""
    dt = p.dt if dt is None else dt
    u1 = u + dt * rhs(u, p, t, s)
    u2 = 0.75 * u + 0.25 * (u1 + dt * rhs(u1, p, t + dt, s))
    u3 = (1.0 / 3.0) * u + (2.0 / 3.0) * (u2 + dt * rhs(u2, p, t + 0.5 * dt, s))
    return u3, t + dt


def step_adaptive(u, p: BurgersParams, t=0.0, s=None, max_substeps=1000):
    """Euler sub-stepping with a global CFL limit; solver_1d.py:148-179.

    Returns (u_new, t_new, substeps)."""
    target = float(p.dt)
    substep = 0
    while target > 0:
        max_u = float(np.max(np.abs(u)))                     # :158 (global max)
        allowed = p.adaptive_CFL * p.dx / max_u if max_u > 0 else target
        dt_local = min(target, allowed)
        u = u + u.dtype.type(dt_local) * rhs(u, p, t, s)
        t = t + dt_local
        target -= dt_local
        if target > 0 and int(math.ceil(target / dt_local)) > max_substeps:   # :173-176
            break
        substep += 1
    return u, t, substep


def rollout(u0, p: BurgersParams, steps, scheme="euler", t0=0.0, s=None):
    """Frames [B, steps, N] of `steps` fixed steps (trainer_1d.py:154-183 with a fixed s)."""
    fn = step_euler if scheme == "euler" else step_ssprk3
    frames = np.empty((u0.shape[0], steps, u0.shape[1]), dtype=u0.dtype)
    u, t = u0, t0
    for k in range(steps):
        u, t = fn(u, p, t, s)
        frames[:, k] = u
    return frames
