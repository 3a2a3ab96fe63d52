"""Seeded synthetic rough surfaces (the workload generator of the benchmarks).

A Gaussian self-affine height field with random phases and an isotropic
power spectrum |h(k)|^2 ~ |k|^(-2(1+H)) on the annulus k_lo <= |k| <= k_hi
(in cycles per domain), zero elsewhere, rescaled to a given RMS; the gap is
g0 = -h (contact starts at the highest summit).  This stands in for the
reference's external surface generator, which is not available here.
"""

import numpy as np


def self_affine_height(Ns, hurst=0.8, rms=0.002, k_lo=4.0, k_hi=64.0, seed=42):
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(Ns, 1.0 / Ns)
    kk = np.hypot(k[:, None], k[None, :])
    amp = np.zeros_like(kk)
    band = (kk >= k_lo) & (kk <= k_hi)
    amp[band] = kk[band] ** (-(1.0 + hurst))  # |h_k| ~ |k|^-(1+H)
    phase = np.exp(2j * np.pi * rng.random((Ns, Ns)))
    h = np.real(np.fft.ifft2(amp * phase))
    h *= rms / h.std()
    return h


def self_affine_gap(Ns, hurst=0.8, rms=0.002, k_lo=4.0, k_hi=64.0, seed=42):
    """Flat (Ns*Ns,) float64 gap g0 = -h."""
    return np.ascontiguousarray((-self_affine_height(Ns, hurst, rms, k_lo, k_hi, seed)).ravel())
