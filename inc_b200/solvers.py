"""Drop-in replacements for the reference 1D solvers, running on B200 kernels.

``BurgersSolverTorch`` and ``KSSolverTorch`` keep the constructor, ``step``
signatures, attributes (``correction_s``, ``correction_u``, ``t``) and errors of
``solvers/solver_1d.py`` in tum-pbs/INC, so ``trainer/trainer_1d.py``'s
``simulate_rollout`` drives them unchanged.  Every step is one launch of a
hand-written sm_100a kernel through the C ABI in ``libinc_b200.so``; autograd
goes through hand-written adjoint kernels (``torch.autograd.Function``).

State tensors must be FP32, contiguous, on a CUDA device.  There is no CPU
path: a missing library raises ``NativeLibraryError``.
"""
from __future__ import annotations

import copy
import ctypes as C
import math

import torch

from . import _native as nat

_SCHEMES = {"euler": nat.INC_TS_EULER, "ssprk3": nat.INC_TS_SSPRK3}


def _check_state(u: torch.Tensor, n: int, what: str = "u") -> None:
    if not isinstance(u, torch.Tensor):
        raise TypeError(f"{what} must be a torch.Tensor")
    if not u.is_cuda:
        raise ValueError(f"{what} must live on a CUDA device (inc_b200 has no CPU path)")
    if u.dtype != torch.float32:
        raise TypeError(f"{what} must be float32 (got {u.dtype})")
    if u.dim() != 2 or u.shape[1] != n:
        raise ValueError(f"{what} must have shape [batch, {n}] (got {tuple(u.shape)})")


def _contig(t):
    return None if t is None else t.contiguous()


def _rows_param(v, rows, device, name):
    """A scalar stays a scalar; a [B], [B,1] tensor becomes a contiguous FP32 [B] tensor."""
    if isinstance(v, torch.Tensor):
        if v.numel() == 1 and rows != 1:
            return float(v.item()), None
        if v.numel() != rows:
            raise ValueError(f"{name} tensor must have shape [batch_size,1]")
        return 0.0, v.detach().reshape(rows).to(device=device, dtype=torch.float32).contiguous()
    return float(v), None


# ----------------------------------------------------------------------------
# Burgers
# ----------------------------------------------------------------------------
class _BurgersLaunch:
    """Everything one Burgers launch needs, with the tensors it points to kept alive."""

    def __init__(self, solver: "BurgersSolverTorch", u: torch.Tensor, t):
        p = solver.param
        rows, n = u.shape
        dev = u.device
        self.dev = dev
        d = nat.BurgersDesc()
        d.rows, d.n = rows, n
        d.scheme = _SCHEMES[solver.time_scheme]
        d.convection = nat.INC_CONV_WENO if p.convection_term == "WENO" else nat.INC_CONV_FDM
        cpt = int(getattr(solver, "cells_per_thread", 0) or 0)
        if cpt == 0:
            cpt = solver._tuned_cpt(n, rows, dev)
        d.cells_per_thread = cpt
        d.dx = float(solver.dx)
        d.dt = float(solver.dt)
        self.keep = []
        nu, nu_rows = _rows_param(solver.nu, rows, dev, "nu")
        d.nu = nu
        d.nu_rows = nat.ptr(nu_rows)
        self.keep.append(nu_rows)
        eq = p.equation_type
        self.t0, self.t_rows = 0.0, None
        self.timed = eq == "learning"  # only the forcing source reads the time
        if eq in ("homogeneous", "viscosity"):
            d.source = nat.INC_SRC_NONE
        elif eq == "linear":
            d.source = nat.INC_SRC_LINEAR
            beta, beta_rows = _rows_param(p.beta, rows, dev, "beta")
            d.beta = beta
            d.beta_rows = nat.ptr(beta_rows)
            self.keep.append(beta_rows)
        elif eq == "learning":
            d.source = nat.INC_SRC_FORCING
            forcing = solver._forcing_pack(rows, dev)
            d.forcing_terms = forcing.shape[-1]
            d.forcing = forcing.data_ptr()
            x = solver._x32(dev)
            d.x = x.data_ptr()
            self.keep += [forcing, x]
            self._bind_time(t, rows)
        else:
            raise ValueError("Unknown equation type.")
        self.desc = d
        self.t_ptr = None if self.t_rows is None else self.t_rows.data_ptr()
        self.dref = C.byref(d)  # the descriptor's address, built once (it keeps d alive)
        self.dev_index = dev.index

    def _bind_time(self, t, rows):
        if isinstance(t, torch.Tensor):
            if t.numel() != rows:
                raise ValueError("t tensor must have shape [batch_size,1]")
            # a snapshot: the solver advances its t in place after the step, and a
            # backward launched later must see the time of this step
            self.t_rows = t.detach().reshape(rows).to(device=self.dev, dtype=torch.float32).clone()
            self.t0 = 0.0
        else:
            self.t0, self.t_rows = float(t), None
        self.t_ptr = None if self.t_rows is None else self.t_rows.data_ptr()

    def at(self, t):
        """This launch at time t: itself when the equation does not read the time, else a
        shallow copy with the time bound (the descriptor and its tensors are shared)."""
        if not self.timed:
            return self
        c = copy.copy(self)
        c._bind_time(t, self.desc.rows)
        return c

    def step(self, u, s, out):
        # the per-step path of the drop-in solver: the bound function, the descriptor's
        # address and the raw stream, and a device switch only when another is current
        idx = self.dev_index
        fn = nat.lib().inc_burgers_step
        sp = None if s is None else s.data_ptr()
        if torch.cuda.current_device() == idx:
            rc = fn(self.dref, u.data_ptr(), sp, self.t_ptr, self.t0, out.data_ptr(), nat.raw_stream(idx))
        else:
            with nat.on_device(self.dev):
                rc = fn(self.dref, u.data_ptr(), sp, self.t_ptr, self.t0, out.data_ptr(), nat.raw_stream(idx))
        if rc:
            nat.check(rc, "inc_burgers_step")

    def step_bwd(self, u, s, g, gu, gs):
        with nat.on_device(self.dev):
            rc = nat.lib().inc_burgers_step_bwd(C.byref(self.desc), u.data_ptr(), nat.ptr(s), nat.ptr(self.t_rows),
                                                self.t0, g.data_ptr(), gu.data_ptr(), nat.ptr(gs),
                                                nat.stream_of(self.dev))
        nat.check(rc, "inc_burgers_step_bwd")

    def rollout(self, u0, s, steps, frames, u_final, ckpt_every, ckpts):
        with nat.on_device(self.dev):
            rc = nat.lib().inc_burgers_rollout(C.byref(self.desc), u0.data_ptr(), nat.ptr(s), nat.ptr(self.t_rows),
                                               self.t0, steps, nat.ptr(frames), nat.ptr(u_final), ckpt_every,
                                               nat.ptr(ckpts), nat.stream_of(self.dev))
        nat.check(rc, "inc_burgers_rollout")

    def cnn_rollout(self, weights, u0, steps, frames, corrections, u_final, ckpt_every=0, ckpts=None, acts=None):
        """The fused CNN-corrected rollout; with ``acts`` ([rows, steps, 2, 32, n] float32) it
        also records the hidden layers' pre-activations for cnn_rollout_bwd."""
        lib = nat.lib()
        args = (C.byref(self.desc), weights.data_ptr(), u0.data_ptr(), nat.ptr(self.t_rows), self.t0, steps,
                nat.ptr(frames), nat.ptr(corrections), nat.ptr(u_final), int(ckpt_every), nat.ptr(ckpts))
        with nat.on_device(self.dev):
            if acts is None:
                rc = lib.inc_burgers_cnn_rollout(*args, nat.stream_of(self.dev))
            else:
                rc = lib.inc_burgers_cnn_rollout_acts(*args, acts.data_ptr(), nat.stream_of(self.dev))
        nat.check(rc, "inc_burgers_cnn_rollout")

    def cnn_rollout_bwd(self, weights, ckpts, corrections, steps, ckpt_every, g_frames, g_corrections, g_final,
                        g_u0, g_weights, work, acts=None):
        """Its backward; ``acts`` (the forward's record) replaces recomputing z2 and z3."""
        lib = nat.lib()
        args = (C.byref(self.desc), weights.data_ptr(), ckpts.data_ptr(), corrections.data_ptr(),
                nat.ptr(self.t_rows), self.t0, steps, ckpt_every, nat.ptr(g_frames), nat.ptr(g_corrections),
                nat.ptr(g_final), g_u0.data_ptr(), g_weights.data_ptr(), work.data_ptr())
        with nat.on_device(self.dev):
            if acts is None:
                rc = lib.inc_burgers_cnn_rollout_bwd(*args, nat.stream_of(self.dev))
            else:
                rc = lib.inc_burgers_cnn_rollout_bwd_acts(*args, acts.data_ptr(), nat.stream_of(self.dev))
        nat.check(rc, "inc_burgers_cnn_rollout_bwd")

    def rollout_bwd(self, ckpts, s, steps, ckpt_every, g_frames, g_final, g_u0, g_s):
        with nat.on_device(self.dev):
            rc = nat.lib().inc_burgers_rollout_bwd(C.byref(self.desc), ckpts.data_ptr(), nat.ptr(s),
                                                   nat.ptr(self.t_rows), self.t0, steps, ckpt_every,
                                                   nat.ptr(g_frames), nat.ptr(g_final), g_u0.data_ptr(),
                                                   nat.ptr(g_s), nat.stream_of(self.dev))
        nat.check(rc, "inc_burgers_rollout_bwd")


class BurgersStepFn(torch.autograd.Function):
    """u_new = step(u, s); backward = the hand-written adjoint kernel."""

    @staticmethod
    def forward(ctx, u, s, launch):
        out = torch.empty_like(u)
        launch.step(u, s, out)
        ctx.launch = launch
        ctx.has_s = s is not None
        ctx.save_for_backward(u, s if s is not None else u.new_empty(0))
        return out

    @staticmethod
    def backward(ctx, g):
        u, s = ctx.saved_tensors
        s = s if ctx.has_s else None
        gu = torch.empty_like(u)
        gs = torch.empty_like(u) if (ctx.has_s and ctx.needs_input_grad[1]) else None
        ctx.launch.step_bwd(u, s, g.contiguous(), gu, gs)
        return gu, gs, None


class BurgersSolverTorch:
    """WENO5-LF / FDM Burgers solver; drop-in for solver_1d.py:44-195.

    ``sim_params`` fields read: resolution, dt, x, adaptive_CFL, L, nu, device,
    convection_term ("WENO"|"FDM"), equation_type ("homogeneous"|"viscosity"|
    "linear"|"learning"), batch_size, beta, J, A, omega, phi, l.  Optional
    extras: ``time_scheme`` ("euler", the reference's integrator and the
    default, or "ssprk3") and ``cells_per_thread`` (kernel shape override).
    """

    def __init__(self, sim_params, LOG=None):
        self.param = sim_params
        self.resolution = sim_params.resolution
        self.dt = sim_params.dt
        self.x = sim_params.x
        self.t = 0.0
        self.adaptive_CFL = sim_params.adaptive_CFL
        self.correction_s = None
        self.L = sim_params.L
        self.nu = sim_params.nu
        self.device = sim_params.device
        self.dx = sim_params.L / sim_params.resolution
        self.LOG = LOG
        if sim_params.convection_term == "FDM":
            self.calc_nonlinear = self.calc_nonlinear_FDM
        elif sim_params.convection_term == "WENO":
            self.calc_nonlinear = self.calc_nonlinear_weno
        else:
            raise ValueError("Convection scheme not recognized")
        self.time_scheme = str(getattr(sim_params, "time_scheme", "euler")).lower()
        if self.time_scheme not in _SCHEMES:
            raise ValueError(f"Unknown time scheme {self.time_scheme!r} (euler | ssprk3)")
        self.cells_per_thread = int(getattr(sim_params, "cells_per_thread", 0) or 0)
        self._forcing_cache = None
        self._x_cache = None
        self._cpt_cache = None
        self._launch_cache = None
        self._d2t = self._d1t = None

    def _tuned_cpt(self, n, rows, dev):
        """Cells per lane from the autotuner cache (0 = library default)."""
        key = (n, rows, self.time_scheme, str(dev))
        if self._cpt_cache is None or self._cpt_cache[0] != key:
            from . import autotune
            self._cpt_cache = (key, autotune.best_burgers(n, rows, self.time_scheme, dev))
        return self._cpt_cache[1]

    # -- parameters packed for the kernels ------------------------------------
    def _forcing_pack(self, rows, dev):
        p = self.param
        objs = (p.A, p.omega, p.phi, p.l)
        key = (rows, str(dev), p.J, p.L) + tuple(getattr(o, "_version", None) for o in objs)
        c = self._forcing_cache
        if c is not None and c[0] == key and all(a is b for a, b in zip(c[2], objs)):
            return c[1]
        J = int(p.J)

        def rj(v):
            v = torch.as_tensor(v, dtype=torch.float64, device=dev)
            return v.reshape(rows, J) if v.numel() == rows * J else v.reshape(1, J).expand(rows, J)

        kx = 2 * math.pi * rj(p.l) / float(p.L)
        pack = torch.stack([rj(p.A), rj(p.omega), rj(p.phi), kx], dim=1).to(torch.float32).contiguous()
        self._forcing_cache = (key, pack, objs)  # holds objs: their ids cannot be reused
        return pack

    def _x32(self, dev):
        if self._x_cache is None or self._x_cache.device != dev:
            self._x_cache = torch.as_tensor(self.x, device=dev).to(torch.float32).reshape(-1).contiguous()
        return self._x_cache

    # -- reference API ------------------------------------------------------------
    def initial_conditions(self, x=None, t=None):
        """Initial condition from the forcing parameters (solver_1d.py:68-72)."""
        x = self.x if x is None else x
        t = self.t if t is None else t
        return self._compute_delta(x, t)

    def _compute_delta(self, x, t):
        """sum_j A_j sin(omega_j t + 2 pi l_j x / L + phi_j) (solver_1d.py:74-85), set-up only."""
        p = self.param
        x_ = torch.as_tensor(x, device=self.device).reshape(1, -1)
        delta = torch.zeros(p.batch_size, x_.shape[1], device=self.device, dtype=x_.dtype)
        t = torch.full((p.batch_size, 1), t, device=self.device) if isinstance(t, (int, float)) else t
        if t.shape != (p.batch_size, 1):
            raise ValueError("t tensor must have shape [batch_size,1]")
        for j in range(p.J):
            arg = p.omega[..., j] * t + (2 * torch.pi * p.l[..., j] / p.L) * x_ + p.phi[..., j]
            delta = delta + p.A[..., j] * torch.sin(arg)
        return delta

    # -- the reference's term methods (solver_1d.py:87-146) -------------------------
    # Each is one launch of inc_burgers_terms on the solver's parameters: the same
    # device arithmetic as the step kernels, each term to its own array.  They are
    # not differentiable here (step() and the rollouts are); under autograd they
    # raise instead of returning a result without a gradient.
    def _terms(self, u, conv=None, want=("nonlinear",)):
        _check_state(u, self.resolution)
        if torch.is_grad_enabled() and u.requires_grad:
            raise RuntimeError("BurgersSolverTorch term methods are not differentiable here; "
                               "differentiate step() or the rollouts instead")
        u = u.contiguous()
        outs = {k: torch.empty_like(u) for k in want}
        if u.shape[0] == 0:
            return outs
        launch = _BurgersLaunch(self, u, self.t)
        d = launch.desc
        if conv is not None:
            d = nat.BurgersDesc.from_buffer_copy(d)
            d.convection = nat.INC_CONV_WENO if conv == "WENO" else nat.INC_CONV_FDM
        with nat.on_device(launch.dev):
            rc = nat.lib().inc_burgers_terms(C.byref(d), u.data_ptr(), nat.ptr(launch.t_rows), launch.t0,
                                             nat.ptr(outs.get("nonlinear")), nat.ptr(outs.get("linear")),
                                             nat.ptr(outs.get("source")), nat.stream_of(launch.dev))
        nat.check(rc, "inc_burgers_terms")
        return outs

    def calc_nonlinear_weno(self, u):
        """-(D- f+ + D- f-)/dx with WENO5 Lax-Friedrichs fluxes (solver_1d.py:129-142)."""
        return self._terms(u, "WENO")["nonlinear"]

    def calc_nonlinear_FDM(self, u):
        """-u D1 u with the periodic central difference (solver_1d.py:125-127)."""
        return self._terms(u, "FDM")["nonlinear"]

    def calc_linear(self, u):
        """nu D2 u (solver_1d.py:144-146); the kernels apply D2 as its three-point stencil."""
        return self._terms(u, want=("linear",))["linear"]

    def _compute_source(self, u):
        """The equation's source term (solver_1d.py:104-114): 0.0 for homogeneous /
        viscosity, beta u for linear, the forcing sum at self.t for learning."""
        eq = self.param.equation_type
        if eq in ("homogeneous", "viscosity"):
            return 0.0
        if eq not in ("linear", "learning"):
            raise ValueError("Unknown equation type.")
        return self._terms(u, want=("source",))["source"]

    def _apply_corrections(self, source):
        """source + correction_s when a correction is set (solver_1d.py:116-123)."""
        if self.correction_s is not None:
            source = source + self.correction_s
        return source

    def _create_diffusion_matrix(self):
        """The dense periodic second-difference matrix / dx^2 (solver_1d.py:95-102).  Only
        for callers that read it: the kernels never form it."""
        n = self.resolution
        i = torch.arange(n, device=self.device)
        m = torch.zeros(n, n, device=self.device)
        m[i, (i - 1) % n] += 1.0 / self.dx ** 2
        m[i, i] += -2.0 / self.dx ** 2
        m[i, (i + 1) % n] += 1.0 / self.dx ** 2
        return m

    def _create_convection_matrix(self):
        """The dense periodic central first-difference matrix (solver_1d.py:87-93)."""
        n = self.resolution
        i = torch.arange(n, device=self.device)
        m = torch.zeros(n, n, device=self.device)
        m[i, (i - 1) % n] += -1.0 / (2 * self.dx)
        m[i, (i + 1) % n] += 1.0 / (2 * self.dx)
        return m

    @property
    def D2_T(self):
        """Transpose of the diffusion matrix (solver_1d.py:58), built on first access."""
        if self._d2t is None:
            self._d2t = self._create_diffusion_matrix().T
        return self._d2t

    @property
    def D1_T(self):
        """Transpose of the convection matrix; the reference defines it for FDM convection
        only (solver_1d.py:61)."""
        if self.param.convection_term != "FDM":
            raise AttributeError("'BurgersSolverTorch' object has no attribute 'D1_T' (WENO convection)")
        if self._d1t is None:
            self._d1t = self._create_convection_matrix().T
        return self._d1t

    def launch_for(self, u, t=None):
        """The kernel configuration of this solver for state u at time t (default self.t)."""
        _check_state(u, self.resolution)
        return _BurgersLaunch(self, u, self.t if t is None else t)

    def _launch_key(self, u):
        p = self.param
        eq = p.equation_type
        static = (u.shape, u.get_device(), self.time_scheme, p.convection_term, eq, self.dt, self.dx,
                  self.cells_per_thread)
        objs = (self.nu,)
        if eq == "linear":
            objs += (p.beta,)
        elif eq == "learning":
            objs += (p.A, p.omega, p.phi, p.l, p.J, p.L, self.x)
        return static, objs, tuple(getattr(o, "_version", None) for o in objs)

    def _cached_launch(self, u):
        """The launch descriptor of the last step, rebuilt only when the shape, the scheme or
        a parameter changes (a parameter tensor replaced by another, or modified in place);
        step() then only binds the time."""
        static, objs, versions = self._launch_key(u)
        c = self._launch_cache
        if (c is not None and c[0] == static and c[2] == versions and len(c[1]) == len(objs)
                and all(a is b or (not isinstance(a, torch.Tensor) and not isinstance(b, torch.Tensor) and a == b)
                        for a, b in zip(c[1], objs))):
            return c[3]
        launch = _BurgersLaunch(self, u, self.t)
        self._launch_cache = (static, objs, versions, launch)  # holds objs: their ids cannot be reused
        return launch

    def step(self, u):
        """Advance by dt (forward Euler, or SSP-RK3 when configured); solver_1d.py:181-195."""
        if self.adaptive_CFL is not None:
            return self.step_adaptive(u)
        _check_state(u, self.resolution)
        u = u.contiguous()
        if u.shape[0] == 0:  # an empty batch: nothing to launch
            self.t += self.dt
            return u.clone()
        launch = self._cached_launch(u).at(self.t)
        s = _contig(self.correction_s)
        if s is not None:
            _check_state(s, self.resolution, "correction_s")
        if torch.is_grad_enabled() and (u.requires_grad or (s is not None and s.requires_grad)):
            u_new = BurgersStepFn.apply(u, s, launch)
        else:
            u_new = torch.empty_like(u)
            launch.step(u, s, u_new)
        self.t += self.dt
        if self.LOG is not None:
            self.LOG.info(f"CFL = {torch.max(torch.abs(u)) * self.dt / self.dx:.2f}, time_step: {self.dt}")
        return u_new

    @property
    def last_substeps(self):
        """Substeps of the last adaptive step (reads the device counter)."""
        subs = getattr(self, "_substeps_dev", None)
        return None if subs is None else int(subs.item())

    def step_adaptive(self, u):
        """Adaptive-CFL sub-stepping (solver_1d.py:148-179), entirely on the GPU."""
        from .adaptive import burgers_step_adaptive
        return burgers_step_adaptive(self, u)


# ----------------------------------------------------------------------------
# Kuramoto-Sivashinsky
# ----------------------------------------------------------------------------
_KS_SCHEMES = {"ETRK2": nat.INC_KS_ETRK2, "ETD1": nat.INC_KS_ETD1}


class KSPlan:
    """Device-side integrator plan: row pairing, FP64-computed coefficients, twiddles."""

    def __init__(self, rows, n, dt, scheme, domain_size_host, device, dealias=False, threads_per_pair=0):
        self.device = torch.device(device)
        size = nat.lib().inc_ks_plan_size(rows, n)
        if size < 0:
            raise ValueError(f"KS resolution must be a power of two in [16, 512] (got {n})")
        self.buf = torch.empty(int(size), dtype=torch.uint8, device=self.device)
        p = nat.KSPlan()
        p.rows, p.n, p.scheme, p.dealias = rows, n, _KS_SCHEMES[scheme], int(bool(dealias))
        p.threads_per_pair, p.dt, p.dev = int(threads_per_pair), float(dt), self.buf.data_ptr()
        host = (C.c_float * rows)(*[float(v) for v in domain_size_host])
        with nat.on_device(self.device):
            rc = nat.lib().inc_ks_plan_init(C.byref(p), host, nat.stream_of(self.device))
        nat.check(rc, "inc_ks_plan_init")
        self.c = p
        self.rows, self.n = rows, n

    def step(self, u, s, cu, out):
        with nat.on_device(self.device):
            rc = nat.lib().inc_ks_step(C.byref(self.c), u.data_ptr(), nat.ptr(s), nat.ptr(cu), out.data_ptr(),
                                       nat.stream_of(self.device))
        nat.check(rc, "inc_ks_step")

    def step_bwd(self, u, s, cu, g, gu, gs):
        with nat.on_device(self.device):
            rc = nat.lib().inc_ks_step_bwd(C.byref(self.c), u.data_ptr(), nat.ptr(s), nat.ptr(cu), g.data_ptr(),
                                           gu.data_ptr(), nat.ptr(gs), nat.stream_of(self.device))
        nat.check(rc, "inc_ks_step_bwd")

    def rollout(self, u0, s, steps, frames, u_final, ckpt_every, ckpts):
        with nat.on_device(self.device):
            rc = nat.lib().inc_ks_rollout(C.byref(self.c), u0.data_ptr(), nat.ptr(s), steps, nat.ptr(frames),
                                          nat.ptr(u_final), ckpt_every, nat.ptr(ckpts), nat.stream_of(self.device))
        nat.check(rc, "inc_ks_rollout")

    def rollout_bwd(self, ckpts, s, steps, ckpt_every, g_frames, g_final, g_u0, g_s, work=None):
        """The rollout's VJP.  ``work`` (default: allocated here) is the device
        scratch of ``rollout_bwd_work_size(ckpt_every)`` bytes in which the
        segment replay keeps the substep states; ``work=False`` rebuilds them
        per step instead (fewer bytes, more transforms)."""
        with nat.on_device(self.device):
            if work is False:
                rc = nat.lib().inc_ks_rollout_bwd(C.byref(self.c), ckpts.data_ptr(), nat.ptr(s), steps, ckpt_every,
                                                  nat.ptr(g_frames), nat.ptr(g_final), g_u0.data_ptr(), nat.ptr(g_s),
                                                  nat.stream_of(self.device))
            else:
                if work is None:
                    work = torch.empty(self.rollout_bwd_work_size(ckpt_every), dtype=torch.uint8, device=self.device)
                rc = nat.lib().inc_ks_rollout_bwd_ws(C.byref(self.c), ckpts.data_ptr(), nat.ptr(s), steps,
                                                     ckpt_every, nat.ptr(g_frames), nat.ptr(g_final),
                                                     g_u0.data_ptr(), nat.ptr(g_s), work.data_ptr(), work.numel(),
                                                     nat.stream_of(self.device))
        nat.check(rc, "inc_ks_rollout_bwd")

    def tape_size(self, steps):
        """Bytes of the tape a tape rollout of `steps` step() calls records."""
        n = int(nat.lib().inc_ks_tape_size(C.byref(self.c), int(steps)))
        if n < 0:
            raise ValueError(f"steps must be positive (got {steps})")
        return n

    def rollout_tape(self, u0, s, steps, frames, u_final, tape):
        """rollout() that also records every step's start and substep states in `tape`
        (a uint8 device tensor of tape_size(steps) bytes) for rollout_bwd_tape."""
        with nat.on_device(self.device):
            rc = nat.lib().inc_ks_rollout_tape(C.byref(self.c), u0.data_ptr(), nat.ptr(s), steps, nat.ptr(frames),
                                               nat.ptr(u_final), tape.data_ptr(), tape.numel(),
                                               nat.stream_of(self.device))
        nat.check(rc, "inc_ks_rollout_tape")

    def rollout_bwd_tape(self, tape, s, steps, g_frames, g_final, g_u0, g_s):
        """The VJP of a tape rollout from its recorded states (no replay)."""
        with nat.on_device(self.device):
            rc = nat.lib().inc_ks_rollout_bwd_tape(C.byref(self.c), tape.data_ptr(), tape.numel(), nat.ptr(s), steps,
                                                   nat.ptr(g_frames), nat.ptr(g_final), g_u0.data_ptr(),
                                                   nat.ptr(g_s), nat.stream_of(self.device))
        nat.check(rc, "inc_ks_rollout_bwd_tape")

    def rollout_bwd_work_size(self, ckpt_every):
        """Bytes of device scratch rollout_bwd uses for this plan and ckpt_every."""
        n = int(nat.lib().inc_ks_rollout_bwd_work_size(C.byref(self.c), int(ckpt_every)))
        if n < 0:
            raise ValueError(f"ckpt_every must be positive (got {ckpt_every})")
        return n


class KSStepFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, s, cu, plan):
        out = torch.empty_like(u)
        plan.step(u, s, cu, out)
        ctx.plan = plan
        ctx.flags = (s is not None, cu is not None)
        e = u.new_empty(0)
        ctx.save_for_backward(u, s if s is not None else e, cu if cu is not None else e)
        return out

    @staticmethod
    def backward(ctx, g):
        u, s, cu = ctx.saved_tensors
        has_s, has_cu = ctx.flags
        s = s if has_s else None
        cu = cu if has_cu else None
        gu = torch.empty_like(u)
        gs = torch.empty_like(u) if (has_s and ctx.needs_input_grad[1]) else None
        ctx.plan.step_bwd(u, s, cu, g.contiguous(), gu, gs)
        gcu = gu if (has_cu and ctx.needs_input_grad[2]) else None
        return gu, gs, gcu, None


class KSSubstepFn(torch.autograd.Function):
    """One ETRK2 / ETD1 substep (etrk2_step / etd1_step) and its adjoint kernel."""

    @staticmethod
    def forward(ctx, u, s, plan):
        out = torch.empty_like(u)
        with nat.on_device(plan.device):
            rc = nat.lib().inc_ks_substep(C.byref(plan.c), u.data_ptr(), nat.ptr(s), out.data_ptr(),
                                          nat.stream_of(plan.device))
        nat.check(rc, "inc_ks_substep")
        ctx.plan, ctx.has_s = plan, s is not None
        ctx.save_for_backward(u, s if s is not None else u.new_empty(0))
        return out

    @staticmethod
    def backward(ctx, g):
        u, s = ctx.saved_tensors
        s = s if ctx.has_s else None
        gu = torch.empty_like(u)
        gs = torch.empty_like(u) if (ctx.has_s and ctx.needs_input_grad[1]) else None
        plan = ctx.plan
        with nat.on_device(plan.device):
            rc = nat.lib().inc_ks_substep_bwd(C.byref(plan.c), u.data_ptr(), nat.ptr(s), g.contiguous().data_ptr(),
                                              gu.data_ptr(), nat.ptr(gs), nat.stream_of(plan.device))
        nat.check(rc, "inc_ks_substep_bwd")
        return gu, gs, None


def _fft_rows(v, mode, out):
    with nat.on_device(v.device):
        rc = nat.lib().inc_ks_fft_rows(v.data_ptr(), out.data_ptr(), v.shape[0], v.shape[1], mode,
                                       nat.stream_of(v.device))
    nat.check(rc, "inc_ks_fft_rows")
    return out


class FFTSquareFn(torch.autograd.Function):
    """FFT(u^2) of each real row (complex [B, N], unnormalised as torch.fft.fft) on the
    row-pair FFT kernel; the backward is 2 u Re(sum_k g_k exp(+2 pi i k j / N)), the
    adjoint of a real row's FFT, on the same kernel."""

    @staticmethod
    def forward(ctx, u):
        u = u.contiguous()
        out = torch.empty(u.shape[0], u.shape[1], 2, device=u.device, dtype=torch.float32)
        _fft_rows(u, 1, out)
        ctx.save_for_backward(u)
        return torch.view_as_complex(out)

    @staticmethod
    def backward(ctx, g):
        u, = ctx.saved_tensors
        gr = torch.view_as_real(g.to(torch.complex64).contiguous())
        re = torch.empty_like(u)
        _fft_rows(gr, 2, re)
        return 2.0 * u * re


class KSSolverTorch:
    """Pseudo-spectral KS solver; drop-in for solver_1d.py:198-288.

    ``sim_params`` fields read: resolution, dt, device, domain_size, alpha,
    time_scheme ("ETRK2"|"ETD1"; unknown names raise KeyError).  ``step(u, L)``
    applies two substeps (the reference's hard-coded doublestep).  Optional
    extras: ``dealias`` (2/3-rule truncation of the nonlinear term; off by
    default, as in the reference whose padding is a no-op) and
    ``threads_per_pair`` (kernel shape override).
    """

    def __init__(self, sim_params):
        self.resolution = sim_params.resolution
        self.dt = sim_params.dt
        self.doublestep = True
        self.device = sim_params.device
        self.domain_size = sim_params.domain_size
        self.alpha = sim_params.alpha
        self.correction_s = None
        self.correction_u = None
        self.fft_indices = torch.fft.fftfreq(self.resolution, d=1.0, device=self.device) * self.resolution
        time_scheme_map = {"ETRK2": self.etrk2, "ETD1": self.etd1}
        self.step = time_scheme_map[sim_params.time_scheme]
        self.time_scheme = sim_params.time_scheme
        self.dealias = bool(getattr(sim_params, "dealias", False))
        self.threads_per_pair = int(getattr(sim_params, "threads_per_pair", 0) or 0)
        self._plan_cache = {}
        self._last = None

    def initial_conditions(self):
        """cos(2 pi x) + alpha sin(2 pi x) + normalised noise (solver_1d.py:214-223), set-up only."""
        domain_size = self.domain_size.unsqueeze(1)
        alpha = self.alpha.unsqueeze(1)
        if len(alpha) != len(domain_size):
            raise ValueError("Length of alpha and domain_size must be the same")
        x = torch.linspace(0, 1, self.resolution, device=self.device)
        u = torch.cos(2 * torch.pi * x) + alpha * torch.sin(2 * torch.pi * x)
        eps = torch.randn_like(u)
        return u + eps / torch.linalg.norm(eps)

    def plan_for(self, u, domain_size, scheme=None):
        """The (cached) device plan for this batch's domain sizes."""
        scheme = scheme or self.time_scheme
        rows = u.shape[0]
        if isinstance(domain_size, torch.Tensor):
            key_obj = (id(domain_size), domain_size._version, domain_size.data_ptr(), rows, scheme)
            if self._last is not None and self._last[0] == key_obj:
                return self._last[1]
            vals = domain_size.detach().reshape(-1).to("cpu", torch.float64).tolist()
        else:
            key_obj = None
            vals = [float(domain_size)] if not hasattr(domain_size, "__len__") else [float(v) for v in domain_size]
        if len(vals) == 1 and rows != 1:
            vals = vals * rows
        if len(vals) != rows:
            raise ValueError(f"domain_size must have {rows} entries (got {len(vals)})")
        key = (rows, self.resolution, scheme, float(self.dt), self.dealias, self.threads_per_pair, u.device,
               tuple(vals))
        plan = self._plan_cache.get(key)
        if plan is None:
            tpp = self.threads_per_pair
            if tpp == 0:
                from . import autotune
                tpp = autotune.best_ks(self.resolution, rows, scheme, u.device)
            plan = KSPlan(rows, self.resolution, self.dt, scheme, vals, u.device, self.dealias, tpp)
            if len(self._plan_cache) > 16:
                self._plan_cache.clear()
            self._plan_cache[key] = plan
        if key_obj is not None:
            self._last = (key_obj, plan)
        return plan

    def _step(self, u, domain_size, scheme):
        _check_state(u, self.resolution)
        u = u.contiguous()
        if u.shape[0] == 0:  # an empty batch: nothing to launch
            return u.clone()
        plan = self.plan_for(u, domain_size, scheme)
        s, cu = _contig(self.correction_s), _contig(self.correction_u)
        if s is not None:
            _check_state(s, self.resolution, "correction_s")
        if cu is not None:
            _check_state(cu, self.resolution, "correction_u")
        needs = torch.is_grad_enabled() and any(t is not None and t.requires_grad for t in (u, s, cu))
        if needs:
            return KSStepFn.apply(u, s, cu, plan)
        out = torch.empty_like(u)
        plan.step(u, s, cu, out)
        return out

    def etrk2(self, u, domain_size):
        """u (+ correction_u), then two ETRK2 substeps (solver_1d.py:285-288)."""
        return self._step(u, domain_size, "ETRK2")

    def etd1(self, u, domain_size):
        """u (+ correction_u), then two ETD1 substeps (solver_1d.py:280-283)."""
        return self._step(u, domain_size, "ETD1")

    # -- the reference's single-substep and term methods (solver_1d.py:225-278) ------
    def _substep(self, u, domain_size, scheme):
        _check_state(u, self.resolution)
        u = u.contiguous()
        if u.shape[0] == 0:
            return u.clone()
        plan = self.plan_for(u, domain_size, scheme)
        s = _contig(self.correction_s)
        if s is not None:
            _check_state(s, self.resolution, "correction_s")
        return KSSubstepFn.apply(u, s, plan)

    def etrk2_step(self, u, domain_size):
        """One ETRK2 substep with correction_s, without correction_u (solver_1d.py:257-278)."""
        return self._substep(u, domain_size, "ETRK2")

    def etd1_step(self, u, domain_size):
        """One ETD1 substep with correction_s, without correction_u (solver_1d.py:242-255)."""
        return self._substep(u, domain_size, "ETD1")

    def calc_linear(self, domain_size):
        """(L, wavenumbers) of solver_1d.py:235-240, complex [B, N]: wavenumbers = i k
        with k = 2 pi fftfreq(N) N / domain_size, L = k^2 - k^4 (= -(ik)^2 - (ik)^4).
        Set-up data, computed with torch on the solver's device."""
        ds = torch.as_tensor(domain_size, device=self.device)
        k = (2 * math.pi) * self.fft_indices / ds.unsqueeze(-1)
        zero = torch.zeros_like(k)
        return torch.complex(k * k - k ** 4, zero), torch.complex(zero, k)

    def calc_nonlinear(self, u, wavenumbers):
        """-0.5 wavenumbers FFT(u^2) (solver_1d.py:225-233; the reference's zero padding in
        physical space changes nothing).  FFT(u^2) runs on the row-pair FFT kernel."""
        _check_state(u, self.resolution)
        return -0.5 * wavenumbers * FFTSquareFn.apply(u)
