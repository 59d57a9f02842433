"""ctypes binding of libinc_b200.so (the C ABI declared in include/inc_b200.h).

The library is the product: there is no Python or CPU fallback.  Importing
this module never needs a GPU; loading the library needs the built .so and
fails loudly (``NativeLibraryError``) if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("INC_B200_LIB", os.path.join(_HERE, "_lib", "libinc_b200.so"))

# status codes and enums (include/inc_b200.h)
INC_OK, INC_E_INVALID, INC_E_UNSUPPORTED, INC_E_LAUNCH, INC_E_NONFINITE = range(5)
INC_TS_EULER, INC_TS_SSPRK3 = 0, 1
INC_CONV_WENO, INC_CONV_FDM = 0, 1
INC_SRC_NONE, INC_SRC_LINEAR, INC_SRC_FORCING = 0, 1, 2
INC_KS_ETRK2, INC_KS_ETD1 = 0, 1

_f = C.POINTER(C.c_float)
_vp = C.c_void_p


class NativeLibraryError(RuntimeError):
    """libinc_b200.so is missing or does not load."""


class BurgersDesc(C.Structure):
    _fields_ = [("rows", C.c_int32), ("n", C.c_int32), ("scheme", C.c_int32), ("convection", C.c_int32),
                ("source", C.c_int32), ("forcing_terms", C.c_int32), ("cells_per_thread", C.c_int32),
                ("reserved", C.c_int32), ("dx", C.c_float), ("dt", C.c_float), ("nu", C.c_float),
                ("beta", C.c_float), ("nu_rows", _vp), ("dt_rows", _vp), ("beta_rows", _vp),
                ("forcing", _vp), ("x", _vp)]


class BurgersRaggedDesc(C.Structure):
    _fields_ = [("rows", C.c_int32), ("scheme", C.c_int32), ("convection", C.c_int32),
                ("warps_per_block", C.c_int32), ("offsets", _vp), ("n_rows", _vp), ("nu_rows", _vp),
                ("dt_rows", _vp), ("dx_rows", _vp), ("order", _vp)]


class KSPlan(C.Structure):
    _fields_ = [("rows", C.c_int32), ("n", C.c_int32), ("scheme", C.c_int32), ("dealias", C.c_int32),
                ("threads_per_pair", C.c_int32), ("npairs", C.c_int32), ("split", C.c_int32),
                ("reserved", C.c_int32), ("dt", C.c_double), ("dev", _vp)]


# name -> (restype, argtypes); the full export list of include/inc_b200.h
SIGNATURES = {
    "inc_version": (C.c_int32, []),
    "inc_last_error_string": (C.c_char_p, []),
    "inc_weno_reconstruct": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "inc_burgers_step": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, _vp, _vp]),
    "inc_burgers_step_bwd": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, _vp, _vp, _vp, _vp]),
    "inc_burgers_rollout": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, C.c_int32, _vp, _vp,
                                      C.c_int32, _vp, _vp]),
    "inc_burgers_rollout_bwd": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, C.c_int32, C.c_int32,
                                          _vp, _vp, _vp, _vp, _vp]),
    "inc_burgers_step_adaptive_work_size": (C.c_int64, [C.c_int32]),
    "inc_burgers_step_adaptive": (C.c_int, [C.POINTER(BurgersDesc), C.c_float, C.c_int32, _vp, _vp, _vp,
                                            C.c_double, _vp, _vp, _vp, _vp, _vp]),
    "inc_burgers_step_adaptive_bwd": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, _vp, C.c_int32,
                                                C.c_int32, _vp, _vp, _vp, _vp, _vp]),
    "inc_burgers_terms": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, C.c_double, _vp, _vp, _vp, _vp]),
    "inc_ks_substep": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, _vp, _vp]),
    "inc_ks_substep_bwd": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, _vp, _vp, _vp, _vp]),
    "inc_ks_fft_rows": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "inc_burgers_ragged_rollout": (C.c_int, [C.POINTER(BurgersRaggedDesc), _vp, C.c_int32, _vp, _vp, C.c_int32,
                                             _vp]),
    "inc_ks_plan_size": (C.c_int64, [C.c_int32, C.c_int32]),
    "inc_ks_plan_init": (C.c_int, [C.POINTER(KSPlan), _vp, _vp]),
    "inc_ks_step": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, _vp, _vp, _vp]),
    "inc_ks_step_bwd": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "inc_ks_rollout": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, C.c_int32, _vp, _vp, C.c_int32, _vp, _vp]),
    "inc_ks_rollout_bwd": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp,
                                     _vp]),
    "inc_ks_rollout_bwd_work_size": (C.c_int64, [C.POINTER(KSPlan), C.c_int32]),
    "inc_ks_rollout_bwd_ws": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp,
                                        _vp, C.c_int64, _vp]),
    "inc_ks_tape_size": (C.c_int64, [C.POINTER(KSPlan), C.c_int32]),
    "inc_ks_rollout_tape": (C.c_int, [C.POINTER(KSPlan), _vp, _vp, C.c_int32, _vp, _vp, _vp, C.c_int64, _vp]),
    "inc_ks_rollout_bwd_tape": (C.c_int, [C.POINTER(KSPlan), _vp, C.c_int64, _vp, C.c_int32, _vp, _vp, _vp, _vp,
                                          _vp]),
    "inc_bench_fma": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp]),
    "inc_energy_spectrum": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, _vp]),
    "inc_spectral_conv1d": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, _vp]),
    "inc_spectral_conv1d_bwd": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          _vp]),
    "inc_bias_gelu": (C.c_int, [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "inc_bias_gelu_bwd": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "inc_burgers_rollout_grad_noalloc": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, C.c_int32,
                                                   C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "inc_burgers_cnn_rollout": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, C.c_int32, _vp, _vp,
                                          _vp, C.c_int32, _vp, _vp]),
    "inc_burgers_cnn_rollout_bwd": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, _vp, C.c_double, C.c_int32,
                                              C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "inc_burgers_cnn_rollout_acts": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, C.c_double, C.c_int32, _vp,
                                               _vp, _vp, C.c_int32, _vp, _vp, _vp]),
    "inc_burgers_cnn_rollout_bwd_acts": (C.c_int, [C.POINTER(BurgersDesc), _vp, _vp, _vp, _vp, C.c_double,
                                                   C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
}
INC_NOALLOC_CKPT_FLOATS = 2 * 1024 * 1024
INC_CNN_WEIGHT_FLOATS = 10657

_lib = None
_lock = threading.Lock()


def lib():
    """The loaded library (loaded once)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise NativeLibraryError(
                    f"{LIB_PATH} not found: build it with `python -m inc_b200.build` "
                    "(inc_b200 has no CPU fallback)")
            try:
                h = C.CDLL(LIB_PATH)
            except OSError as e:  # pragma: no cover - depends on the box
                raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(h, name)
                fn.restype = res
                fn.argtypes = args
            _lib = h
    return _lib


def last_error() -> str:
    msg = lib().inc_last_error_string()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    """Raise the Python exception matching an INC status code."""
    if rc == INC_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc in (INC_E_INVALID, INC_E_UNSUPPORTED):
        raise ValueError(msg)
    raise RuntimeError(msg)


def ptr(t) -> int | None:
    """Device pointer of a tensor (or None)."""
    return None if t is None else t.data_ptr()


def raw_stream(idx: int) -> int:
    """The raw cudaStream_t of torch's current stream on device index `idx`."""
    import torch
    raw = getattr(torch._C, "_cuda_getCurrentRawStream", None)
    return raw(idx) if raw is not None else torch.cuda.current_stream(idx).cuda_stream


def stream_of(device) -> int:
    """The raw cudaStream_t of torch's current stream on `device`."""
    import torch
    idx = device.index if isinstance(device, torch.device) else device
    if idx is None:
        idx = torch.cuda.current_device()
    raw = getattr(torch._C, "_cuda_getCurrentRawStream", None)
    return raw(idx) if raw is not None else torch.cuda.current_stream(idx).cuda_stream


class on_device:
    """Make `device` current for a launch (a no-op when it already is)."""

    __slots__ = ("idx", "prev")

    def __init__(self, device):
        self.idx = device.index

    def __enter__(self):
        import torch
        cur = torch.cuda.current_device()
        self.prev = None if (self.idx is None or cur == self.idx) else cur
        if self.prev is not None:
            torch.cuda.set_device(self.idx)
        return self

    def __exit__(self, *exc):
        if self.prev is not None:
            import torch
            torch.cuda.set_device(self.prev)
        return False
