"""B200-native (sm_100a) INC 1D hybrid time-stepper.

Drop-in solvers for tum-pbs/INC's 1D path (solvers/solver_1d.py): WENO5-LF /
FDM Burgers with forward Euler or SSP-RK3, and the pseudo-spectral
Kuramoto-Sivashinsky ETRK2 / ETD1 step, each with the neural correction s(u)
as a source term, hand-written adjoints, fused rollouts and ragged batches.
"""
from .solvers import BurgersSolverTorch, KSSolverTorch  # noqa: F401

__all__ = ["BurgersSolverTorch", "KSSolverTorch"]
__version__ = "0.1.0"
