"""The C-ABI library builds, loads without a GPU and exports every symbol of
include/inc_b200.h; the ctypes structures match the C layout (CPU)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "inc_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(inc_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from inc_b200 import build, _native
    build.build()
    return _native.lib()


def test_header_lists_entry_points():
    names = header_functions()
    assert "inc_burgers_step" in names and "inc_ks_rollout_bwd" in names and len(names) >= 15


def test_library_exports_every_declared_symbol(lib):
    from inc_b200 import _native
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (inc_[a-z0-9_]+)\b", out))
    missing = [n for n in header_functions() if n not in exported]
    assert not missing, missing
    assert set(_native.SIGNATURES) == set(header_functions())


def test_version_and_error_string(lib):
    assert lib.inc_version() == 100
    assert isinstance(lib.inc_last_error_string(), bytes)


def test_argument_checks_need_no_gpu(lib):
    """Invalid descriptors are rejected on the host before any CUDA call."""
    from inc_b200 import _native as nat
    d = nat.BurgersDesc()
    d.rows, d.n, d.dx = 0, 64, 0.1
    assert lib.inc_burgers_step(C.byref(d), None, None, None, 0.0, None, None) == nat.INC_E_INVALID
    d.rows, d.scheme = 2, 7
    assert lib.inc_burgers_step(C.byref(d), None, None, None, 0.0, None, None) == nat.INC_E_INVALID
    assert b"scheme" in lib.inc_last_error_string()
    d.scheme, d.convection = 0, 5
    assert lib.inc_burgers_step(C.byref(d), None, None, None, 0.0, None, None) == nat.INC_E_INVALID
    assert b"Convection" in lib.inc_last_error_string()
    assert lib.inc_weno_reconstruct(None, None, 1, 64, 0, None) == nat.INC_E_INVALID
    assert lib.inc_ks_plan_size(4, 96) == -1
    assert lib.inc_ks_plan_size(4, 64) > 0
    p = nat.KSPlan()
    assert lib.inc_ks_step(C.byref(p), None, None, None, None, None) == nat.INC_E_INVALID


def test_struct_layouts():
    from inc_b200 import _native as nat
    assert C.sizeof(nat.BurgersDesc) == 8 * 4 + 4 * 4 + 5 * 8
    assert C.sizeof(nat.KSPlan) == 8 * 4 + 8 + 8
    assert C.sizeof(nat.BurgersRaggedDesc) == 4 * 4 + 6 * 8


def test_ks_rollout_bwd_work_size_needs_no_gpu(lib):
    """The KS backward's scratch size: one [ckpt_every][3][n] complex slot per
    launched row-pair group (two for the warp-specialised form: ETRK2, 32 lanes and
    up to 8 values per lane), computed on the host from the plan's shape."""
    from inc_b200 import _native as nat
    p = nat.KSPlan()
    p.rows, p.n, p.npairs, p.threads_per_pair, p.scheme = 1024, 256, 512, 32, nat.INC_KS_ETD1
    # 512 pairs of 32 lanes launch one group per 32-thread block: 512 groups
    assert lib.inc_ks_rollout_bwd_work_size(C.byref(p), 8) == 512 * 3 * 8 * 256 * 8
    p.scheme = nat.INC_KS_ETRK2  # the replay runs one segment ahead: two slots per pair
    assert lib.inc_ks_rollout_bwd_work_size(C.byref(p), 8) == 2 * 512 * 3 * 8 * 256 * 8
    assert lib.inc_ks_rollout_bwd_work_size(C.byref(p), 0) == -1
    p.threads_per_pair = 64  # a pair spans two warps, one group per block
    assert lib.inc_ks_rollout_bwd_work_size(C.byref(p), 4) == 512 * 3 * 4 * 256 * 8
    p.npairs = 0  # not initialised
    assert lib.inc_ks_rollout_bwd_work_size(C.byref(p), 8) == -1
    # the scratch entry point rejects a missing or short scratch before any CUDA call
    p.npairs = 512
    assert lib.inc_ks_rollout_bwd_ws(C.byref(p), None, None, 1, 8, None, None, None, None, None, 0,
                                     None) == nat.INC_E_INVALID


def test_new_entry_points_check_arguments_without_gpu(lib):
    """Sizes and argument checks of the tape, adaptive, term and substep entry points,
    all decided on the host before any CUDA call."""
    from inc_b200 import _native as nat
    p = nat.KSPlan()
    p.rows, p.n, p.npairs, p.threads_per_pair = 1024, 256, 512, 32
    # the tape: 4 complex [n] states per row pair and step, row pairs rounded up to 32
    assert lib.inc_ks_tape_size(C.byref(p), 400) == 512 * 400 * 4 * 256 * 8
    p.npairs = 513
    assert lib.inc_ks_tape_size(C.byref(p), 2) == 544 * 2 * 4 * 256 * 8
    assert lib.inc_ks_tape_size(C.byref(p), 0) == -1
    assert lib.inc_ks_rollout_bwd_tape(C.byref(p), None, 0, None, 2, None, None, None, None, None) \
        == nat.INC_E_INVALID
    # adaptive CFL: the work buffer holds a 64-byte control block and two doubles per substep
    assert lib.inc_burgers_step_adaptive_work_size(1000) >= 64 + 16 * 1001
    assert lib.inc_burgers_step_adaptive_work_size(0) == -1
    d = nat.BurgersDesc()
    d.rows, d.n, d.dx, d.dt = 2, 64, 0.1, 0.01
    fake = C.c_void_p(256)  # never dereferenced: the call is rejected before any launch
    assert lib.inc_burgers_step_adaptive(C.byref(d), 0.2, 1000, fake, None, None, 0.0, fake, None, None, None,
                                         None) == nat.INC_E_INVALID
    assert b"work" in lib.inc_last_error_string()
    d.scheme = nat.INC_TS_SSPRK3
    assert lib.inc_burgers_step_adaptive(C.byref(d), 0.2, 1000, fake, None, None, 0.0, fake, None, fake, None,
                                         None) == nat.INC_E_INVALID  # forward Euler only
    # terms and spectra
    d.scheme, d.rows = nat.INC_TS_EULER, 0
    assert lib.inc_burgers_terms(C.byref(d), fake, None, 0.0, None, None, None, None) == nat.INC_E_INVALID
    assert lib.inc_ks_fft_rows(fake, fake, 4, 64, 3, None) == nat.INC_E_INVALID
    assert lib.inc_ks_fft_rows(fake, fake, 4, 96, 1, None) == nat.INC_E_UNSUPPORTED
    p.npairs = 0
    assert lib.inc_ks_substep(C.byref(p), fake, None, fake, None) == nat.INC_E_INVALID
