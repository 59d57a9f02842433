"""The allocation-free Burgers rollout gradient entry point (GPU).

inc_burgers_rollout_grad_noalloc serves callers that may not allocate device
memory while the op runs (a host framework owning all device memory, or a
fixed memory budget): it keeps the rollout checkpoints in a fixed array inside
the library.  Its results must equal those of the allocating pair
inc_burgers_rollout + inc_burgers_rollout_bwd, on two calls in a row (the
second call reuses the array the first one filled).  This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C
import math

import pytest
import torch

pytestmark = pytest.mark.gpu


def _desc(nat, rows, n, dt, nu, scheme):
    d = nat.BurgersDesc()
    d.rows, d.n = rows, n
    d.scheme = nat.INC_TS_SSPRK3 if scheme == "ssprk3" else nat.INC_TS_EULER
    d.convection, d.source = nat.INC_CONV_WENO, nat.INC_SRC_NONE
    d.dx, d.dt, d.nu = 2 * math.pi / n, dt, nu
    return d


def _inputs(rows, n, steps, seed, dev):
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.arange(n, dtype=torch.float64) * (2 * math.pi / n)
    a = torch.rand(rows, 3, generator=g, dtype=torch.float64) - 0.5
    u0 = sum(a[:, k:k + 1] * torch.sin((k + 1) * x + k) for k in range(3)).float()
    s = 0.05 * torch.randn(rows, n, generator=g)
    gf = torch.randn(rows, steps, n, generator=g)
    gl = torch.randn(rows, n, generator=g)
    return [t.to(dev).contiguous() for t in (u0, s, gf, gl)]


def _allocating(lib, nat, d, u0, s, gf, gl, steps, k, stream):
    rows, n = u0.shape
    frames = torch.empty(rows, steps, n, device=u0.device)
    ckpts = torch.empty(rows, (steps + k - 1) // k, n, device=u0.device)
    g_u0, g_s = torch.empty_like(u0), torch.empty_like(u0)
    nat.check(lib.inc_burgers_rollout(C.byref(d), u0.data_ptr(), s.data_ptr(), None, 0.0, steps, frames.data_ptr(),
                                      None, k, ckpts.data_ptr(), stream), "rollout")
    nat.check(lib.inc_burgers_rollout_bwd(C.byref(d), ckpts.data_ptr(), s.data_ptr(), None, 0.0, steps, k,
                                          gf.data_ptr(), gl.data_ptr(), g_u0.data_ptr(), g_s.data_ptr(), stream),
              "rollout_bwd")
    return frames, g_u0, g_s


def _noalloc(lib, nat, d, u0, s, gf, gl, steps, k, stream):
    rows, n = u0.shape
    frames = torch.empty(rows, steps, n, device=u0.device)
    u_final = torch.empty_like(u0)
    g_u0, g_s = torch.empty_like(u0), torch.empty_like(u0)
    nat.check(lib.inc_burgers_rollout_grad_noalloc(C.byref(d), u0.data_ptr(), s.data_ptr(), None, 0.0, steps, k,
                                                   gf.data_ptr(), gl.data_ptr(), frames.data_ptr(),
                                                   u_final.data_ptr(), g_u0.data_ptr(), g_s.data_ptr(), stream),
              "rollout_grad_noalloc")
    return frames, u_final, g_u0, g_s


def _rel(a, b):
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def test_noalloc_matches_allocating_entry_points_twice(cuda):
    from inc_b200 import _native as nat
    lib = nat.lib()
    stream = nat.stream_of(cuda)
    # different problems in a row: each call reuses the area the previous one filled.  At most
    # 148 rows take the one-row-per-CTA kernels, more rows the warp-per-row ones.
    for call, (rows, n, steps, k, scheme, seed) in enumerate([(64, 256, 40, 8, "ssprk3", 1),
                                                               (37, 128, 29, 5, "euler", 2),
                                                               (300, 256, 16, 8, "ssprk3", 3)]):
        d = _desc(nat, rows, n, 0.004, 0.01, scheme)
        u0, s, gf, gl = _inputs(rows, n, steps, seed, cuda)
        fr_a, gu_a, gs_a = _allocating(lib, nat, d, u0, s, gf, gl, steps, k, stream)
        fr_b, uf_b, gu_b, gs_b = _noalloc(lib, nat, d, u0, s, gf, gl, steps, k, stream)
        torch.cuda.synchronize()
        assert torch.equal(fr_a, fr_b), call
        assert torch.equal(uf_b, fr_a[:, -1]), call
        assert _rel(gu_b, gu_a) < 1e-6, call
        assert _rel(gs_b, gs_a) < 1e-6, call


def test_noalloc_rejects_oversized_problem(cuda):
    from inc_b200 import _native as nat
    lib = nat.lib()
    rows, n, steps, k = 4096, 512, 8, 8  # 4096 * 1 * 512 = 2M floats: fits
    d = _desc(nat, rows + 1, n, 0.004, 0.01, "euler")  # one row more: over the limit
    u0 = torch.zeros(rows + 1, n, device=cuda)
    g = torch.empty_like(u0)
    rc = lib.inc_burgers_rollout_grad_noalloc(C.byref(d), u0.data_ptr(), None, None, 0.0, steps, k, None, None,
                                              None, None, g.data_ptr(), None, nat.stream_of(cuda))
    assert rc == nat.INC_E_INVALID
    assert "checkpoint area" in nat.last_error()
    assert rows * ((steps + k - 1) // k) * n == nat.INC_NOALLOC_CKPT_FLOATS
