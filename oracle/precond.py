"""13-tap stencil and full-grid |k| Fourier preconditioners (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  Both apply
z = Pi_C W Pi_C g on the contact set C: centre g over C, apply W, keep z on C
and remove its contact mean (fourier_precond.cpp:32-49).
"""

import numpy as np

from .operators import rfft2, irfft2


def kernel_grid(Nw):
    """w = F^-1 |k| (DC zeroed) on an Nw^2 periodic grid, normalised by w(0,0).

    stencil_precond.cpp:19-43.  Returned as an (Nw, Nw) array [iy, ix].
    """
    nh = Nw // 2 + 1
    ky = np.arange(Nw)
    kof = np.where(ky < Nw // 2, ky, ky - Nw).astype(np.float64)
    kx = np.arange(nh, dtype=np.float64)
    C = np.hypot(kx[None, :], kof[:, None]).astype(np.complex128)
    C[0, 0] = 0.0
    G = irfft2(C, (Nw, Nw))
    return G / G[0, 0]


class StencilPreconditioner:
    """Truncated real-space kernel of |k| on the l2 disc |d| <= R.

    Constructor stencil_precond.cpp:199-220; apply :63-109.
    """

    def __init__(self, Ns, radius=2):
        if radius < 1:
            raise ValueError("stencil radius must be >= 1")
        if 2 * radius + 1 > Ns:
            raise ValueError("stencil radius too large for the grid")
        self.Ns = int(Ns)
        self.R = int(radius)
        Nw = Ns if Ns < 512 else 512
        w = kernel_grid(Nw)
        dx, dy, ww = [], [], []
        for ddy in range(-radius, radius + 1):
            for ddx in range(-radius, radius + 1):
                if ddx * ddx + ddy * ddy > radius * radius:
                    continue
                dx.append(ddx)
                dy.append(ddy)
                ww.append(float(w[ddy % Nw, ddx % Nw]))
        self.tap_dx, self.tap_dy, self.tap_w = dx, dy, ww

    def ntaps(self):
        return len(self.tap_w)

    def apply(self, g, contact, dtype=None):
        Ns = self.Ns
        g = np.asarray(g)
        dtype = np.dtype(g.dtype if dtype is None else dtype).type
        c = np.asarray(contact).astype(bool).reshape(Ns, Ns)
        g2 = g.reshape(Ns, Ns)
        ng = int(c.sum())
        gsum = float(np.sum(g2[c].astype(np.float64)))
        gmean = gsum / ng if ng else 0.0
        gc = np.where(c, g2.astype(np.float64) - gmean, 0.0)
        acc = np.zeros((Ns, Ns), dtype=np.float64)
        for ddx, ddy, w in zip(self.tap_dx, self.tap_dy, self.tap_w):
            # fetch(ix + dx, iy + dy) with periodic wrap
            acc = acc + w * np.roll(gc, shift=(-ddy, -ddx), axis=(0, 1))
        z = np.where(c, acc.astype(dtype), dtype(0)).astype(dtype)
        nc = ng
        if nc:
            zsum = float(np.sum(acc[c]))
            zmean = dtype(zsum / nc)
            z[c] = z[c] - zmean
        return z.reshape(-1)


class FourierPreconditioner:
    """Full-grid FFT application of the |k|/Ns^2 symbol (float table).

    fourier_precond.cpp:12-28 (symbol) and :50-116 (apply_t).
    """

    def __init__(self, Ns):
        self.Ns = int(Ns)
        self.nh = self.Ns // 2 + 1
        norm = np.float32(1.0) / (np.float32(Ns) * np.float32(Ns))
        ky = np.arange(self.Ns)
        kof = np.where(ky < self.Ns // 2, ky, ky - self.Ns).astype(np.float32)
        kx = np.arange(self.nh).astype(np.float32)
        wh = (norm * np.hypot(kx[None, :], kof[:, None])).astype(np.float32)
        wh[0, 0] = np.float32(0.0)
        self.wh = wh

    def apply(self, g, contact, dtype=None):
        Ns = self.Ns
        g = np.asarray(g)
        dtype = np.dtype(g.dtype if dtype is None else dtype).type
        g2 = g.reshape(Ns, Ns).astype(dtype, copy=False)
        c = np.asarray(contact).astype(bool).reshape(Ns, Ns)
        ng = int(c.sum())
        gsum = float(np.sum(g2[c].astype(np.float64)))
        gmean = dtype(gsum / ng) if ng else dtype(0)
        G = np.where(c, g2 - gmean, dtype(0)).astype(dtype)
        C = rfft2(G)
        C *= self.wh.astype(dtype)
        G = irfft2(C, (Ns, Ns)).astype(dtype, copy=False)
        z = np.where(c, G, dtype(0)).astype(dtype)
        nc = ng
        if nc:
            zsum = float(np.sum(G[c].astype(np.float64)))
            zmean = dtype(zsum / nc)
            z[c] = z[c] - zmean
        return z.reshape(-1)
