"""Algorithmic work per cell-step, the numerators of the roofline fractions.

A cell-step is one grid point advanced by one reference ``step()`` call (for
KS: two ETRK2/ETD1 substeps, the reference's doublestep).  Counts are of the
algorithm, not of this implementation's instructions; a divide or a square
root counts as one flop, an FMA as two.

Burgers WENO5-LF right-hand side, per cell (solver_1d.py:4-42, :129-146):
  two WENO5 reconstructions at 70 flops each (3 candidate polynomials 15,
  3 smoothness indicators 36, 3 weights 9, normalised combination 10) = 140;
  flux splitting 8; flux differences 6; diffusion stencil 5; alpha max 1;
  source add 5 -> 165.  Euler step = 165 + 2; SSP-RK3 = 3 * 165 + 8.

KS, the frozen count of the reference algorithm (the roofline numerator):
per substep five complex length-N FFT-class ops (FFT(u^2), IFFT, FFT(u_i^2),
IFFT and FFT(s), solver_1d.py:257-278) at 5 log2 N flops per cell each, plus
~45 pointwise flops; one step() is two substeps: 2 (25 log2 N + 45) = 490 at
N = 256, 540 at N = 512.  ETD1 by the same rule has four FFT-class ops and ~20
pointwise flops per substep (solver_1d.py:242-255).

KS, this implementation's own count (reported beside it): two rows share one
complex FFT and s is transformed once per launch, so a substep is four real
FFTs at 2.5 N log2 N flops each -> 10 log2 N per cell, plus 12 pointwise:
2 (10 log2 N + 12) = 184 at N = 256 (ETD1: 2 (5 log2 N + 8)).

Bytes per cell-step (FP32): a step() launch reads u and writes u' (8 B) and
reads s when present (+4 B); a fused rollout writes one frame per step (4 B)
and reads its inputs once.
"""
from __future__ import annotations

import math

BURGERS_RHS_FLOPS = 165
BURGERS_FLOPS = {"euler": BURGERS_RHS_FLOPS + 2, "ssprk3": 3 * BURGERS_RHS_FLOPS + 8}


def ks_flops_per_cell_step(n: int, scheme: str = "ETRK2") -> float:
    """Reference-algorithm flops per cell-step (the roofline numerator)."""
    lg = math.log2(n)
    sub = (25 * lg + 45) if scheme == "ETRK2" else (20 * lg + 20)
    return 2 * sub


def ks_impl_flops_per_cell_step(n: int, scheme: str = "ETRK2") -> float:
    """Flops per cell-step this implementation executes (row pairs share one FFT)."""
    lg = math.log2(n)
    sub = (10 * lg + 12) if scheme == "ETRK2" else (5 * lg + 8)
    return 2 * sub


def plain_bytes_per_cell_step(with_s: bool) -> int:
    return 8 + (4 if with_s else 0)


FUSED_BYTES_PER_CELL_STEP = 4

# Periodic CNN corrector (Conv1d 1 -> 32 -> 32 -> 32 -> 1, kernel 5) per cell:
# 2 * (32*5 + 2 * 32*32*5 + 32*5) multiply-adds-as-two = 21,120 flops (bias and
# GELU not counted), evaluated once per step before the solver step.
CNN_FLOPS_PER_CELL = 2 * (32 * 5 + 2 * 32 * 32 * 5 + 32 * 5)


def burgers_cnn_flops_per_cell_step(scheme: str = "ssprk3") -> int:
    return CNN_FLOPS_PER_CELL + BURGERS_FLOPS[scheme]
