"""Pin the numpy oracle against golden vectors produced by the reference itself (CPU)."""
import numpy as np
import pytest

from oracle import burgers as ob
from oracle import ks as oks
from tests.golden_io import burgers_case, ks_case, load, rel_l2

BZ = load("burgers_golden.npz")
KZ = load("ks_golden.npz")


def test_weno_reconstruction_matches_reference():
    f = BZ["weno_f"]
    assert np.allclose(ob.weno_reconstruction(f, "left"), BZ["weno_left"], rtol=1e-13, atol=1e-13)
    assert np.allclose(ob.weno_reconstruction(f, "right"), BZ["weno_right"], rtol=1e-13, atol=1e-13)
    with pytest.raises(ValueError):
        ob.weno_reconstruction(f, "up")


def test_burgers_terms_match_reference():
    u = BZ["op_u"]
    dx = 2 * np.pi / u.shape[1]
    assert rel_l2(ob.nonlinear_weno(u, dx), BZ["op_nonlinear_weno"]) < 1e-13
    assert rel_l2(ob.linear(u, 0.01, dx), BZ["op_linear"]) < 1e-13


@pytest.mark.parametrize("name", [str(n) for n in BZ["cases"]])
def test_burgers_rollouts_match_reference(name):
    p, u0, t0, s, scheme = burgers_case(BZ, name)
    frames = BZ[f"{name}.frames"]
    u, t = u0, t0
    for k in range(frames.shape[1]):
        if p.adaptive_CFL is not None:
            u, t, n = ob.step_adaptive(u, p, t, s)
        elif scheme == "rk3":
            u, t = ob.step_ssprk3(u, p, t, s)
        else:
            u, t = ob.step_euler(u, p, t, s)
        assert rel_l2(u, frames[:, k]) < 1e-12, (name, k)
    if p.adaptive_CFL is not None:
        assert n == int(BZ[f"{name}.substeps"])


def _burgers_loss(p, u0, t0, s, scheme, w):
    u, t, acc = u0, t0, 0.0
    for k in range(w.shape[1]):
        u, t = (ob.step_ssprk3 if scheme == "rk3" else ob.step_euler)(u, p, t, s)
        acc += float((u * w[:, k]).sum())
    return acc


@pytest.mark.parametrize("name", [str(n) for n in BZ["grad_cases"]])
def test_burgers_reference_gradients_match_oracle_fd(name):
    """Golden autograd gradients (reference, FP64) vs central FD of the oracle."""
    p, u0, t0, s, scheme = burgers_case(BZ, name)
    w = BZ[f"{name}.w"]
    assert abs(_burgers_loss(p, u0, t0, s, scheme, w) - float(BZ[f"{name}.loss"])) < 1e-10
    rng = np.random.default_rng(7)
    h = 1e-6
    for _ in range(3):
        du, ds_ = rng.standard_normal(u0.shape), rng.standard_normal(s.shape)
        fd_u = (_burgers_loss(p, u0 + h * du, t0, s, scheme, w) - _burgers_loss(p, u0 - h * du, t0, s, scheme, w)) / (2 * h)
        fd_s = (_burgers_loss(p, u0, t0, s + h * ds_, scheme, w) - _burgers_loss(p, u0, t0, s - h * ds_, scheme, w)) / (2 * h)
        assert abs(fd_u - float((BZ[f"{name}.grad_u"] * du).sum())) < 1e-6 * max(1.0, abs(fd_u))
        assert abs(fd_s - float((BZ[f"{name}.grad_s"] * ds_).sum())) < 1e-6 * max(1.0, abs(fd_s))


@pytest.mark.parametrize("name", [str(n) for n in KZ["cases"]])
def test_ks_rollouts_match_reference(name):
    c = ks_case(KZ, name)
    frames = KZ[f"{name}.frames"]
    u = c["u0"]
    for k in range(frames.shape[1]):
        u = oks.step(u, c["L"], c["dt"], c["scheme"], c["s"], c["cu"])
        assert rel_l2(u, frames[:, k]) < 1e-12, (name, k)
    sub = oks.etrk2_step if c["scheme"] == "ETRK2" else oks.etd1_step
    assert rel_l2(sub(c["u0"], c["L"], c["dt"], c["s"]), KZ[f"{name}.substep"]) < 1e-12


def _ks_loss(c, u0, s, w):
    u, acc = u0, 0.0
    for k in range(w.shape[1]):
        u = oks.step(u, c["L"], c["dt"], c["scheme"], s)
        acc += float((u * w[:, k]).sum())
    return acc


@pytest.mark.parametrize("name", [str(n) for n in KZ["grad_cases"]])
def test_ks_reference_gradients_match_oracle_fd(name):
    c = ks_case(KZ, name)
    w = KZ[f"{name}.w"]
    u0, s = c["u0"], c["s"]
    assert abs(_ks_loss(c, u0, s, w) - float(KZ[f"{name}.loss"])) < 1e-9
    rng = np.random.default_rng(11)
    h = 1e-6
    for _ in range(3):
        du, ds_ = rng.standard_normal(u0.shape), rng.standard_normal(s.shape)
        fd_u = (_ks_loss(c, u0 + h * du, s, w) - _ks_loss(c, u0 - h * du, s, w)) / (2 * h)
        fd_s = (_ks_loss(c, u0, s + h * ds_, w) - _ks_loss(c, u0, s - h * ds_, w)) / (2 * h)
        assert abs(fd_u - float((KZ[f"{name}.grad_u"] * du).sum())) < 1e-6 * max(1.0, abs(fd_u))
        assert abs(fd_s - float((KZ[f"{name}.grad_s"] * ds_).sum())) < 1e-6 * max(1.0, abs(fd_s))


def test_ks_unknown_scheme_raises_keyerror():
    with pytest.raises(KeyError):
        oks.step(np.zeros((1, 8)), [8.0], 0.1, "RK4")


def test_ks_dealias_padding_is_identity():
    """The reference's 3/2 physical-space padding squares u exactly (no dealiasing)."""
    rng = np.random.default_rng(0)
    u = rng.standard_normal((2, 16))
    padded = np.concatenate([u, np.zeros((2, 8))], axis=1) ** 2
    assert np.array_equal(padded[:, :16], u ** 2)
