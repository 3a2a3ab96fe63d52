"""Free-space (zero-padded Love) and doubly periodic operators (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  Layout follows the
reference: a field is flat ``iy*Ns + ix``; here it is viewed as an (Ns, Ns)
array indexed [iy, ix], and half spectra as [ky, kx] with kx in [0, n/2]
(the reference's ``C(kx, ky)`` with kx contiguous).  All transforms are
unnormalised like ``src/fft_engine.hpp:20-23``: forward with scipy's
``norm="backward"`` (no scale) and inverse with ``norm="forward"`` (no scale).
"""

import os

import numpy as np
import scipy.fft as sfft

from .love import boussinesq_table

# Threads for scipy's pocketfft.  The reference threads its transforms with
# OpenMP slabs (fft_engine.hpp:147-221); the oracle uses every host core.
WORKERS = int(os.environ.get("ORACLE_FFT_WORKERS", os.cpu_count() or 1))


def rfft2(a):
    return sfft.rfft2(a, workers=WORKERS)


def irfft2(c, shape):
    return sfft.irfft2(c, s=shape, norm="forward", workers=WORKERS)


class FFTOperator:
    """Exact free-space convolution with the Love table on a (2Ns)^2 grid.

    fft_operator.cpp:18-69 (build) and :87-138 (matvec).  Kh is the real
    half spectrum of the wrap-around embedded table with 1/M^2 folded in.
    """

    def __init__(self, Ns, L=1.0, E_star=1.0):
        self.Ns = int(Ns)
        self.M = 2 * self.Ns
        self.nh = self.Ns + 1
        self.L = float(L)
        self.E_star = float(E_star)
        self.table = boussinesq_table(self.Ns, self.L, self.E_star)
        self.build()
        self.Kh_f = None

    def build(self):
        Ns, M = self.Ns, self.M
        # embed: offset d >= 0 at index d, d < 0 at M + d; row/col Ns zero
        # (fft_operator.cpp:31-44)
        idx = np.arange(M)
        d = np.where(idx < Ns, idx, idx - M)
        valid = idx != Ns
        ad = np.abs(d)
        K = self.table[ad[:, None].clip(0, Ns - 1), ad[None, :].clip(0, Ns - 1)]
        K = np.where(valid[:, None] & valid[None, :], K, 0.0)
        Kc = rfft2(K)
        max_im = np.max(np.abs(Kc.imag))
        max_re = np.max(np.abs(Kc.real))
        if max_im > 1e-10 * max_re:  # fft_operator.cpp:48-61
            raise RuntimeError("FFTOperator: kernel spectrum has a "
                               "non-negligible imaginary part")
        self.max_im_ratio = max_im / max_re
        self.Kh = Kc.real * (1.0 / (float(M) * float(M)))  # [ky, kx], (M, nh)

    def build_single_caches(self):
        if self.Kh_f is None:
            self.Kh_f = self.Kh.astype(np.float32)

    def matvec(self, x, dtype=np.float64):
        """u = S x; scatter -> r2c -> * Kh -> c2r -> gather (:87-138)."""
        Ns, M = self.Ns, self.M
        x = np.asarray(x)
        if x.size != Ns * Ns:
            raise ValueError("FFTOperator::matvec: x size != Ns*Ns")
        if dtype == np.float32:
            self.build_single_caches()
            Kh = self.Kh_f
        else:
            Kh = self.Kh
        G = np.zeros((M, M), dtype=dtype)
        G[:Ns, :Ns] = x.reshape(Ns, Ns)
        C = rfft2(G)
        C *= Kh
        y = irfft2(C, (M, M))
        return np.ascontiguousarray(y[:Ns, :Ns]).reshape(-1).astype(dtype, copy=False)


class PeriodicFFTOperator:
    """u_hat(q) = 2 p_hat / (E* |q|), zero mode 0: periodic_fft_operator.cpp."""

    def __init__(self, Ns, L=1.0, E_star=1.0):
        if Ns < 2:
            raise ValueError("grid_size must be at least 2")
        if not L > 0.0:
            raise ValueError("domain_size must be positive")
        if not E_star > 0.0:
            raise ValueError("E_star must be positive")
        self.Ns = int(Ns)
        self.nh = self.Ns // 2 + 1
        self.scale = L / (np.pi * E_star * float(self.Ns) * self.Ns)  # :11-24
        ky = np.arange(self.Ns)
        my = np.where(ky < (self.Ns + 1) // 2, ky, ky - self.Ns).astype(np.float64)
        kx = np.arange(self.nh, dtype=np.float64)
        m2 = kx[None, :] * kx[None, :] + (my * my)[:, None]
        with np.errstate(divide="ignore"):
            w = np.where(m2 > 0.0, self.scale / np.sqrt(m2), 0.0)  # :34-47
        self.symbol = w
        self.symbol_f = w.astype(np.float32)

    def build_single_caches(self):
        pass

    def matvec(self, x, dtype=np.float64):
        Ns = self.Ns
        x = np.asarray(x)
        if x.size != Ns * Ns:
            raise ValueError("PeriodicFFTOperator input size mismatch")
        w = self.symbol_f if dtype == np.float32 else self.symbol
        C = rfft2(x.reshape(Ns, Ns).astype(dtype, copy=False))
        C *= w
        return irfft2(C, (Ns, Ns)).reshape(-1).astype(dtype, copy=False)
