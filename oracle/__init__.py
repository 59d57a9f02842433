"""CPU oracle for the INC 1D hybrid time-stepper (test infrastructure only).

This package restates, in numpy, the reference's 1D solvers
(``solvers/solver_1d.py`` of tum-pbs/INC) so that the CUDA path in ``inc_b200``
can be checked against it.  It is the *checker*, never the product: only the
test suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference
arm import it.  Nothing in ``inc_b200`` imports this package, and the product
path fails loudly when its CUDA library is missing instead of falling back here.

Every function is dtype-generic: pass float64 arrays for the FP64 oracle (the
parity reference) and float32 arrays for the CPU baseline (the reference runs
its solvers in FP32 on torch).

Pinning: the reference ships no tests, fixtures or golden vectors for this
path.  The restatement is pinned against golden vectors that
``tests/golden/make_golden.py`` produced by importing the reference's own
``solvers/solver_1d.py`` (FP64, with the one-line ``_apply_corrections`` call fix
described in ``oracle.burgers``) and running it on seeded inputs.
"""

from . import burgers, ks  # noqa: F401
