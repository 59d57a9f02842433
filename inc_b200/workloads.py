"""Seeded synthetic inputs for the benchmark configurations.

The reference's INC_Data trajectories are not available, so every workload is
generated here in FP64 from a fixed seed and cast to FP32:

* burgers_plain_config  - N=128, B=32, nu=0.01, dt=0.01, 200 steps, s=0,
  u0 = sum_{k=1..5} A_k sin(k x + phi_k), A ~ U[-0.5, 0.5], phi ~ U[0, 2 pi)
* ks_plain_config       - N=256, B=1024, L=64, dt=0.25, 400 step() calls,
  u0 = sum_{k=1..8} a_k cos(2 pi k x / L + phi_k), a_k ~ N(0,1)/k,
  s = a constant N(0, 0.01^2) field per trajectory
* burgers_batched_config- 4096 rows, N ~ U{64,128,256,512}, nu log-uniform in
  [1e-3, 5e-2], u0 as above, dt = 0.4 min(dx / max|u0|, dx^2 / nu), 500 steps
* burgers_diff_config   - N=256, B=256, nu=0.01, 32-step unroll
* ks_diff_config        - L=100, N=512, B=512, dt=0.2, 64-step unroll
"""
from __future__ import annotations

import math

import numpy as np


def sines_u0(rng, B, N, L=2 * math.pi, K=5):
    x = np.arange(N) * (L / N)
    a = rng.uniform(-0.5, 0.5, (B, K))
    ph = rng.uniform(0, 2 * math.pi, (B, K))
    k = np.arange(1, K + 1)
    return (a[:, :, None] * np.sin(k[None, :, None] * x[None, None, :] * (2 * math.pi / L)
                                   + ph[:, :, None])).sum(1)


def ks_u0(rng, B, N, L, K=8):
    x = np.arange(N) * (L / N)
    k = np.arange(1, K + 1)
    a = rng.standard_normal((B, K)) / k
    ph = rng.uniform(0, 2 * math.pi, (B, K))
    return (a[:, :, None] * np.cos(2 * math.pi * k[None, :, None] * x[None, None, :] / L
                                   + ph[:, :, None])).sum(1)


def burgers_plain_config(seed=0, B=32, N=128, steps=200):
    rng = np.random.default_rng(seed)
    return dict(name="burgers_plain", B=B, N=N, L=2 * math.pi, nu=0.01, dt=0.01, steps=steps,
                u0=sines_u0(rng, B, N), scheme="ssprk3")


def ks_plain_config(seed=1, B=1024, N=256, L=64.0, dt=0.25, steps=400):
    rng = np.random.default_rng(seed)
    return dict(name="ks_plain", B=B, N=N, L=L, dt=dt, steps=steps, scheme="ETRK2",
                u0=ks_u0(rng, B, N, L), s=0.01 * rng.standard_normal((B, N)))


def burgers_batched_config(seed=2, rows=4096, steps=500, ns=(64, 128, 256, 512)):
    rng = np.random.default_rng(seed)
    L = 2 * math.pi
    n_rows = rng.choice(np.asarray(ns), size=rows)
    nu = np.exp(rng.uniform(math.log(1e-3), math.log(5e-2), rows))
    u0, dt, dx = [], [], []
    for n, v in zip(n_rows, nu):
        u = sines_u0(rng, 1, int(n))[0]
        h = L / n
        u0.append(u)
        dx.append(h)
        dt.append(0.4 * min(h / max(np.abs(u).max(), 1e-12), h * h / v))
    return dict(name="burgers_batched", rows=rows, steps=steps, n=n_rows, nu=nu, dt=np.asarray(dt),
                dx=np.asarray(dx), u0=u0, scheme="ssprk3")


def burgers_diff_config(seed=3, B=256, N=256, steps=32):
    rng = np.random.default_rng(seed)
    return dict(name="burgers_diff", B=B, N=N, L=2 * math.pi, nu=0.01, dt=0.01, steps=steps,
                u0=sines_u0(rng, B, N), scheme="ssprk3", ckpt_every=8)


def ks_diff_config(seed=4, B=512, N=512, L=100.0, dt=0.2, steps=64):
    rng = np.random.default_rng(seed)
    return dict(name="ks_diff", B=B, N=N, L=L, dt=dt, steps=steps, scheme="ETRK2", u0=ks_u0(rng, B, N, L),
                ckpt_every=8)
