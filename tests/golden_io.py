"""Readers for the committed golden vectors (tests/golden/*.npz)."""
import os

import numpy as np

from oracle import burgers as ob

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def burgers_case(z, name):
    """(params, u0, t0, s or None, scheme) for a Burgers golden case."""
    g = lambda k: z[f"{name}.{k}"]  # noqa: E731
    nu = g("nu")
    cfl = float(g("cfl"))
    p = ob.BurgersParams(resolution=int(g("N")), L=float(g("L")), dt=float(g("dt")),
                         nu=(nu if nu.ndim else float(nu)), convection_term=str(g("conv")),
                         equation_type=str(g("eq")), beta=g("beta"), A=g("A"), omega=g("omega"),
                         phi=g("phi"), l=g("l"), x=g("x"),
                         adaptive_CFL=(None if np.isnan(cfl) else cfl))
    s = g("s")
    return p, g("u0"), g("t0"), (s if s.size else None), str(g("scheme"))


def ks_case(z, name):
    g = lambda k: z[f"{name}.{k}"]  # noqa: E731
    s = g("s")
    out = dict(scheme=str(g("scheme")), N=int(g("N")), L=g("L"), dt=float(g("dt")), u0=g("u0"),
               s=(s if s.size else None))
    if f"{name}.cu" in z:
        cu = g("cu")
        out["cu"] = cu if cu.size else None
    return out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
