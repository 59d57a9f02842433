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

KS ETRK2 substep, per cell (solver_1d.py:257-278): four real FFTs of length N
(FFT(u^2), IFFT, FFT(ui^2), IFFT) at 2.5 N log2 N flops each (half the
5 N log2 N of a complex FFT) -> 10 log2 N; pointwise work 12 (two squares,
and per half-spectrum bin the multipliers of stage 1 and 2).  One step() is
two substeps.  ETD1 substep: two real FFTs -> 5 log2 N + 8.

Bytes per cell-step (FP32): a step() launch reads u and writes u' (8 B) and
reads s when present (+4 B); a fused rollout writes one frame per step (4 B)
and reads its inputs once.
"""
from __future__ import annotations

import math

BURGERS_RHS_FLOPS = 165
BURGERS_FLOPS = {"euler": BURGERS_RHS_FLOPS + 2, "ssprk3": 3 * BURGERS_RHS_FLOPS + 8}


def ks_flops_per_cell_step(n: int, scheme: str = "ETRK2") -> float:
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
