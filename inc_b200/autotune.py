"""Kernel-shape autotuner for the Burgers and KS kernels.

The free kernel parameters are the row layout across lanes: cells per lane
(Burgers, 1 / 2 with one row per CTA, or 4 / 8 / 16 with a row inside a warp) and lanes per row pair (KS,
4..64).  Narrow layouts give more instruction-level parallelism per lane and win
on large batches; wide layouts give more warps per row and win on small
batches.  ``tune_burgers`` / ``tune_ks`` time every valid layout on the current
GPU for one (kind, n, batch bucket, scheme) and store the winner; the solvers
read the winner through ``best_burgers`` / ``best_ks`` when their sim_params do
not force a layout.

Cache: JSON at ``$INC_B200_AUTOTUNE_CACHE`` (default
``~/.cache/inc_b200/autotune.json``), keyed by GPU name, kind, n, batch bucket
(next power of two) and scheme.  Set ``INC_B200_AUTOTUNE=1`` to tune lazily on
the first use of a key (the tuning launches run once, outside any capture).
"""
from __future__ import annotations

import json
import os
import threading

import torch

BURGERS_CPT = (1, 2, 4, 8, 16)
KS_TPP = (4, 8, 16, 32, 64)
KS_SHAPES = {(4, 4), (4, 8), (4, 16), (8, 8), (4, 32), (8, 16), (8, 32), (16, 16), (16, 32), (32, 16),
             (4, 64), (8, 64)}

_lock = threading.Lock()
_cache = None


def cache_path() -> str:
    return os.environ.get("INC_B200_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "inc_b200", "autotune.json"))


def _load():
    global _cache
    if _cache is None:
        try:
            with open(cache_path()) as f:
                _cache = json.load(f)
        except (OSError, ValueError):
            _cache = {}
    return _cache


def _save():
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"  # one per process: ranks of a multi-GPU run tune concurrently
        with open(tmp, "w") as f:
            json.dump(_cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: keep the in-memory table


def bucket(rows: int) -> int:
    b = 1
    while b < rows:
        b <<= 1
    return b


_names = {}


def _device_name(device) -> str:
    idx = torch.device(device).index if device is not None else None
    if idx not in _names:
        _names[idx] = torch.cuda.get_device_name(device) if torch.cuda.is_available() else "cpu"
    return _names[idx]


def key(kind: str, n: int, rows: int, scheme: str, device=None) -> str:
    return f"{_device_name(device)}|{kind}|n{n}|b{bucket(rows)}|{scheme}"


def burgers_candidates(n: int):
    """Warp layouts (4/8/16 cells per lane, 2..32 lanes per row) and, for n >= 64,
    the one-row-per-CTA layouts (1/2 cells per lane, up to 512 lanes)."""
    if not (8 <= n <= 512 and n & (n - 1) == 0):
        return []
    warp_lanes = {4: (2, 32), 8: (4, 32), 16: (8, 32)}  # lanes per row with kernels built
    out = []
    for c in BURGERS_CPT:
        if c <= 2:
            if n >= 64 and n // c <= 512:
                out.append(c)
        elif warp_lanes[c][0] <= n // c <= warp_lanes[c][1]:
            out.append(c)
    return out


def ks_candidates(n: int):
    return [t for t in KS_TPP if n % t == 0 and (n // t, t) in KS_SHAPES]


def _time(fn, iters=5):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(iters):
        a.record()
        fn()
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def tune_burgers(n, rows, scheme="ssprk3", convection="WENO", device="cuda", steps=50):
    """Time every cells-per-lane layout on a fused rollout; store and return the best."""
    from types import SimpleNamespace
    from .solvers import BurgersSolverTorch
    dev = torch.device(device)
    g = torch.Generator(device="cpu").manual_seed(0)
    u0 = (0.5 * torch.randn(rows, n, generator=g)).to(dev)
    frames = torch.empty(rows, steps, n, device=dev)
    times = {}
    for cpt in burgers_candidates(n):
        sp = SimpleNamespace(resolution=n, dt=1e-3, x=None, adaptive_CFL=None, L=6.283185307179586, nu=0.01,
                             device=dev, convection_term=convection, equation_type="viscosity", batch_size=rows,
                             time_scheme=scheme, cells_per_thread=cpt)
        launch = BurgersSolverTorch(sp).launch_for(u0)
        times[cpt] = _time(lambda: launch.rollout(u0, None, steps, frames, None, 0, None))
    best = min(times, key=times.get)
    with _lock:
        _load()[key("burgers", n, rows, scheme, dev)] = {"cells_per_thread": best, "ms": times}
        _save()
    return best, times


def tune_ks(n, rows, scheme="ETRK2", device="cuda", steps=50, L=64.0, dt=0.25):
    """Time every lanes-per-pair layout on a fused rollout; store and return the best."""
    from types import SimpleNamespace
    from .solvers import KSSolverTorch
    dev = torch.device(device)
    g = torch.Generator(device="cpu").manual_seed(0)
    u0 = (0.5 * torch.randn(rows, n, generator=g)).to(dev)
    ds = torch.full((rows,), float(L), device=dev)
    frames = torch.empty(rows, steps, n, device=dev)
    times = {}
    for tpp in ks_candidates(n):
        sp = SimpleNamespace(resolution=n, dt=dt, device=dev, domain_size=ds, alpha=torch.zeros(rows, device=dev),
                             time_scheme=scheme, threads_per_pair=tpp)
        plan = KSSolverTorch(sp).plan_for(u0, ds)
        times[tpp] = _time(lambda: plan.rollout(u0, None, steps, frames, None, 0, None))
    best = min(times, key=times.get)
    with _lock:
        _load()[key("ks", n, rows, scheme, dev)] = {"threads_per_pair": best, "ms": times}
        _save()
    return best, times


def tune_ragged(rb, steps=100, margin=0.02):
    """Time the persistent ragged launch at a few grid sizes and keep the fastest on `rb`.
    The default grid (sized to the work) is kept unless another one is faster by more
    than `margin`: launches of a few hundred microseconds differ by about that much from
    run to run, and a pick made on that noise does not carry over to long rollouts."""
    sms = torch.cuda.get_device_properties(rb.device).multi_processor_count
    default = rb.default_grid()
    times = {}
    for g in sorted({default, 2 * sms, 3 * sms, 4 * sms}):
        rb.grid_blocks = g
        times[g] = _time(lambda: rb.rollout(steps))
    best = min(times, key=times.get)
    rb.grid_blocks = best if times[best] < (1.0 - margin) * times[default] else default
    return rb.grid_blocks, times


def best_burgers(n, rows, scheme, device) -> int:
    """Cached cells-per-lane for this problem, or 0 (library default)."""
    with _lock:
        e = _load().get(key("burgers", n, rows, scheme, device))
    if e is not None:
        return int(e["cells_per_thread"])
    if os.environ.get("INC_B200_AUTOTUNE") == "1" and burgers_candidates(n):
        return tune_burgers(n, rows, scheme, device=device)[0]
    return 0


def best_ks(n, rows, scheme, device) -> int:
    """Cached lanes-per-pair for this problem, or 0 (library default)."""
    with _lock:
        e = _load().get(key("ks", n, rows, scheme, device))
    if e is not None:
        return int(e["threads_per_pair"])
    if os.environ.get("INC_B200_AUTOTUNE") == "1" and ks_candidates(n):
        return tune_ks(n, rows, scheme, device=device)[0]
    return 0
