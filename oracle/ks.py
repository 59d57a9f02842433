"""Numpy restatement of the reference Kuramoto-Sivashinsky solver (test infrastructure only).

Follows ``KSSolverTorch`` in ``solvers/solver_1d.py`` of tum-pbs/INC (cited per
function).  u: [B, N] real rows on a periodic domain of length ``domain_size[b]``.
Works in the dtype of its inputs (float64 -> complex128 oracle, float32 ->
complex64 like the reference's torch run).

Facts of the reference kept here on purpose:
* ``calc_nonlinear`` pads u with zeros in physical space to 3N/2, squares and
  truncates back to N (solver_1d.py:225-233), which is exactly ``u**2``: no
  dealiasing happens.
* ``step`` is a double step: ``doublestep = True`` (solver_1d.py:202), so one
  ``step(u, L)`` applies two ETD1 or ETRK2 substeps of ``dt`` (:280-288).
* ``correction_u`` is added once before the two substeps; ``correction_s``
  enters stage 1 of every substep (:251, :271, :281, :286).
"""
from __future__ import annotations

import numpy as np


def _cdtype(dtype):
    return np.complex64 if np.dtype(dtype) == np.float32 else np.complex128


def linear_operator(domain_size, n, dtype=np.float64):
    """(L, wavenumbers) of solver_1d.py:208-210 and :235-240.

    wavenumbers = 2 pi i fftfreq(N) N / domain_size, L = -wn^2 - wn^4 (complex
    dtype, real-valued).  Shapes [B, N]."""
    idx = (np.fft.fftfreq(n, d=1.0) * n).astype(dtype)
    ds = np.asarray(domain_size, dtype=dtype).reshape(-1, 1)
    wn = (2j * np.pi * idx.astype(_cdtype(dtype))) / ds
    wn = wn.astype(_cdtype(dtype))
    lop = -wn ** 2 - wn ** 4
    return lop, wn


def etd_coefficients(lop, dt, scheme="ETRK2"):
    """exp(L dt), phi1, phi2 of solver_1d.py:243-246 (ETD1) and :258-267 (ETRK2)."""
    e = np.exp(lop * dt)
    with np.errstate(divide="ignore", invalid="ignore"):
        if scheme == "ETD1":
            phi1 = np.where(lop == 0, dt * np.ones_like(lop), (e - 1) / lop)
            phi2 = None
        else:
            small = np.abs(lop) < 1e-6
            phi1 = np.where(small, dt * np.ones_like(lop), (e - 1) / lop)
            phi2 = np.where(small, (dt / 2) * np.ones_like(lop), (e - 1 - lop * dt) / (lop ** 2 * dt))
    return e, phi1, phi2


def nonlinear(u, wn):
    """-0.5 * wn * FFT(u^2); solver_1d.py:225-233 (the 3/2 zero padding is a no-op)."""
    return -0.5 * wn * np.fft.fft(u * u, axis=-1)


def etd1_step(u, domain_size, dt, s=None, coeffs=None):
    """solver_1d.py:242-255."""
    lop, wn = linear_operator(domain_size, u.shape[-1], u.dtype)
    e, phi1, _ = coeffs if coeffs is not None else etd_coefficients(lop, dt, "ETD1")
    u_hat = np.fft.fft(u, axis=-1)
    n_hat = nonlinear(u, wn)
    s_hat = np.fft.fft(s, axis=-1) if s is not None else 0.0
    return np.fft.ifft(e * u_hat + phi1 * (n_hat + s_hat), axis=-1).real.astype(u.dtype)


def etrk2_step(u, domain_size, dt, s=None, coeffs=None):
    """solver_1d.py:257-278."""
    lop, wn = linear_operator(domain_size, u.shape[-1], u.dtype)
    e, phi1, phi2 = coeffs if coeffs is not None else etd_coefficients(lop, dt, "ETRK2")
    u_hat = np.fft.fft(u, axis=-1)
    n1 = nonlinear(u, wn)
    s_hat = np.fft.fft(s, axis=-1) if s is not None else 0.0
    ui_hat = e * u_hat + phi1 * (n1 + s_hat)
    ui = np.fft.ifft(ui_hat, axis=-1).real.astype(u.dtype)
    n2 = nonlinear(ui, wn)
    return np.fft.ifft(ui_hat + phi2 * (n2 - n1), axis=-1).real.astype(u.dtype)


def step(u, domain_size, dt, scheme="ETRK2", s=None, cu=None, coeffs=None):
    """One reference ``step(u, L)``: two substeps; solver_1d.py:280-288."""
    if scheme not in ("ETRK2", "ETD1"):      # time_scheme_map lookup, :211-212
        raise KeyError(scheme)
    if cu is not None:
        u = u + cu
    sub = etrk2_step if scheme == "ETRK2" else etd1_step
    u = sub(u, domain_size, dt, s, coeffs)
    return sub(u, domain_size, dt, s, coeffs)


def coefficients_fp64(domain_size, n, dt, scheme="ETRK2", dtype=np.float32):
    """FP64-computed integrator coefficients, rounded to ``dtype``'s complex type.

    Same formulas as ``etd_coefficients``; used to run an FP32 state with FP64
    precomputed coefficients."""
    lop, _ = linear_operator(domain_size, n, np.float64)
    e, p1, p2 = etd_coefficients(lop, dt, scheme)
    c = _cdtype(dtype)
    return e.astype(c), p1.astype(c), (None if p2 is None else p2.astype(c))


def rollout(u0, domain_size, dt, steps, scheme="ETRK2", s=None, coeffs=None):
    """Frames [B, steps, N] of `steps` reference step() calls with a fixed s."""
    frames = np.empty((u0.shape[0], steps, u0.shape[1]), dtype=u0.dtype)
    u = u0
    for k in range(steps):
        u = step(u, domain_size, dt, scheme, s, None, coeffs)
        frames[:, k] = u
    return frames
