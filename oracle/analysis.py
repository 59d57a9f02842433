"""Numpy restatement of the reference's KS energy spectrum (test infrastructure only).

analysis/Plot_KS.py:196-235 of tum-pbs/INC: |FFT(u)|^2 over the first
D//2+1 bins (D even) or (D+1)//2 (D odd), bins 1..-2 (even) or 1.. (odd)
doubled; physical wavenumbers 2 pi k, one row per batch entry."""
import numpy as np


def energy_spectrum(velocity):
    v = np.asarray(velocity)
    if v.ndim == 2:
        v = v[None]
    B, T, D = v.shape
    e = np.abs(np.fft.fft(v.astype(np.float64), axis=-1)) ** 2
    n = D // 2 + 1 if D % 2 == 0 else (D + 1) // 2
    spec = e[..., :n].copy()
    if D % 2 == 0:
        spec[..., 1:-1] *= 2
    else:
        spec[..., 1:] *= 2
    k = 2 * np.pi * np.arange(n, dtype=np.float64) / np.ones((B, 1))
    return spec, k
