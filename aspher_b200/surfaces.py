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


def self_affine_gap_device(Ns, hurst=0.8, rms=0.002, k_lo=4.0, k_hi=64.0, seed=42,
                           device="cuda"):
    """self_affine_gap synthesised on the device (for grids whose host-side
    synthesis would take tens of GB): the same random phases (drawn on the
    host from the same seed) and spectrum; the inverse FFT and the scaling
    run in torch on `device`.  Returns a flat FP64 device tensor, equal to
    self_affine_gap's array up to FFT rounding."""
    import torch
    rng = np.random.default_rng(seed)
    ph = torch.from_numpy(rng.random((Ns, Ns))).to(device)
    k = torch.fft.fftfreq(Ns, 1.0 / Ns, dtype=torch.float64, device=device)
    kk = torch.hypot(k[:, None], k[None, :])
    band = (kk >= k_lo) & (kk <= k_hi)
    amp = torch.where(band, kk.clamp_min(1e-300) ** (-(1.0 + hurst)), torch.zeros_like(kk))
    del kk, band
    spec = torch.polar(amp, 2 * np.pi * ph)
    del amp, ph
    h = torch.fft.ifft2(spec).real
    del spec
    h *= rms / h.std(correction=0)
    return (-h).reshape(-1).contiguous()
