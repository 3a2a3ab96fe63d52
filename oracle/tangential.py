"""Cerruti kernel and the tangential FFT operator (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  Restates, vectorised
over numpy arrays:

* ``cerruti_uxx`` / ``cerruti_uxy`` / ``cerruti_ylog`` --
  ``src/cerruti_kernel.cpp:1-112`` (the element-integrated Cerruti brackets:
  the stable asinh form of ylog with its multipole branch past 1500 max(a, b),
  the u_xx bracket as (1-nu) Love + nu ylog, the rationalised mixed bracket);
* ``CerrutiKernel`` -- ``src/cerruti_kernel.cpp:114-128`` and
  ``include/cerruti_kernel.hpp:35-61`` (xx and xy tables for |dx|, |dy| <
  Ns, yy the x<->y transpose of xx, xy odd in each axis and exactly 0 on the
  axes; prefactors 1/(pi E* (1-nu)) and nu times it);
* ``TangentialFFTOperator`` -- ``src/tangential_operator.cpp:18-140``
  (three tables embedded in wrap-around order on the (2Ns)^2 grid, r2c,
  realness check 1e-10, the 1/M^2 scale folded in; matvec: two padded
  transforms, the all-real 2x2 mix, two inverse transforms, the origin block).
"""

import numpy as np

from .love import _term, love_uz
from .operators import irfft2, rfft2

# cerruti_kernel.cpp:41 (in units of max(a, b))
CERRUTI_FAR_SWITCH = 1500.0


def cerruti_ylog(x_abs, y_abs, a, b):
    """Integral of (x - xi)^2 / rho^3 over the cell (cerruti_kernel.cpp:43-68)."""
    x_abs, y_abs, a, b = np.broadcast_arrays(*(np.asarray(v, np.float64)
                                               for v in (x_abs, y_abs, a, b)))
    mmax = np.where(a > b, a, b)
    r2 = x_abs * x_abs + y_abs * y_abs
    far = r2 > (CERRUTI_FAR_SWITCH * mmax) ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.sqrt(r2)
        r3 = r2 * r
        r5 = r3 * r2
        r7 = r5 * r2
        A = 4.0 * a * b
        x2, y2 = x_abs * x_abs, y_abs * y_abs
        far_val = A * (x2 / r3 + (a * a / 6.0) * (2.0 / r3 - 15.0 * x2 / r5 + 15.0 * x2 * x2 / r7)
                       + (b * b / 6.0) * (-3.0 * x2 / r5 + 15.0 * x2 * y2 / r7))
    k, l = x_abs + a, x_abs - a
    m, n = y_abs + b, y_abs - b
    da = 2.0 * a
    near_val = _term(m, k, l, da) + _term(n, l, k, -da)
    return np.where(far, far_val, near_val)


def cerruti_uxx(x, y, a, b, nu):
    """(1 - nu) Love + nu ylog (cerruti_kernel.cpp:70-79)."""
    xa = np.abs(np.asarray(x, np.float64))
    ya = np.abs(np.asarray(y, np.float64))
    out = (1.0 - nu) * love_uz(xa, ya, a, b) + nu * cerruti_ylog(xa, ya, a, b)
    return out if np.ndim(out) else float(out)


def cerruti_uxy(x, y, a, b):
    """Integral of (x - xi)(y - eta) / rho^3 over the cell, odd in x and y,
    in the rationalised form (cerruti_kernel.cpp:81-112)."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    xa, ya = np.abs(x), np.abs(y)
    k, l = xa + a, xa - a
    m, n = ya + b, ya - b
    Rkm, Rkn = np.hypot(k, m), np.hypot(k, n)
    Rlm, Rln = np.hypot(l, m), np.hypot(l, n)
    num = 16.0 * a * b * xa * ya * (1.0 / (Rkn + Rln) + 1.0 / (Rkm + Rlm))
    den = (Rlm + Rln) * (Rkn + Rkm)
    with np.errstate(divide="ignore", invalid="ignore"):
        mag = np.where(den > 0.0, num / den, 0.0)
    sx = np.where(x >= 0.0, 1.0, -1.0)
    sy = np.where(y >= 0.0, 1.0, -1.0)
    out = sx * sy * mag
    return out if np.ndim(out) else float(out)


class CerrutiKernel:
    """Tangential influence tables of an Ns x Ns grid of square cells."""

    def __init__(self, Ns, L=1.0, E_star=1.0, nu=0.3):
        self.Ns = int(Ns)
        self.L, self.E_star, self.nu = float(L), float(E_star), float(nu)
        self.h = self.L / self.Ns
        self.a = 0.5 * self.h
        self.pref = 1.0 / (np.pi * self.E_star * (1.0 - self.nu))
        self.prefnu = self.nu * self.pref
        d = np.arange(self.Ns, dtype=np.float64) * self.h
        # [dy, dx] for dx, dy >= 0 (cerruti_kernel.cpp:120-127)
        self.xx = self.pref * cerruti_uxx(d[None, :], d[:, None], self.a, self.a, self.nu)
        self.xy = self.prefnu * cerruti_uxy(d[None, :], d[:, None], self.a, self.a)

    def offsets(self, dx, dy):
        """(xx, yy, xy) at signed integer offsets (cerruti_kernel.hpp:44-58);
        0 outside (-Ns, Ns)."""
        dx = np.asarray(dx)
        dy = np.asarray(dy)
        ax, ay = np.abs(dx), np.abs(dy)
        inside = (ax < self.Ns) & (ay < self.Ns)
        cx, cy = np.clip(ax, 0, self.Ns - 1), np.clip(ay, 0, self.Ns - 1)
        xx = np.where(inside, self.xx[cy, cx], 0.0)
        yy = np.where(inside, self.xx[cx, cy], 0.0)
        sgn = np.where((dx > 0) == (dy > 0), 1.0, -1.0)
        xy = np.where(inside & (dx != 0) & (dy != 0), sgn * self.xy[cy, cx], 0.0)
        return xx, yy, xy

    def assemble_dense(self):
        """[[XX, XY], [XY, YY]] (cerruti_kernel.cpp:130-146)."""
        N = self.Ns * self.Ns
        i = np.arange(N)
        ix, iy = i % self.Ns, i // self.Ns
        dix = ix[:, None] - ix[None, :]
        diy = iy[:, None] - iy[None, :]
        xx, yy, xy = self.offsets(dix, diy)
        return np.block([[xx, xy], [xy, yy]])


class TangentialFFTOperator:
    """u = C q, q = [q_x; q_y] and u = [u_x; u_y] stacked (N each)."""

    def __init__(self, kernel):
        self.k = kernel
        self.Ns = kernel.Ns
        self.M = 2 * self.Ns
        self.build()

    def build(self):
        Ns, M = self.Ns, self.M
        idx = np.arange(M)
        d = np.where(idx < Ns, idx, idx - M)  # wrap-around offsets
        valid = idx != Ns
        DX, DY = np.meshgrid(d, d)  # [iy, ix]
        xx, yy, xy = self.k.offsets(DX, DY)
        mask = valid[:, None] & valid[None, :]
        norm = 1.0 / (M * M)
        self.spectra = {}
        for name, t in (("xx", xx), ("yy", yy), ("xy", xy)):
            c = rfft2(np.where(mask, t, 0.0))
            max_im = np.max(np.abs(c.imag))
            max_re = np.max(np.abs(c.real))
            if max_im > 1e-10 * max_re:
                raise RuntimeError("TangentialFFTOperator: %s spectrum parity broken" % name)
            self.spectra[name] = norm * c.real
        self.max_im_ratio = None

    def matvec(self, q, dtype=np.float64):
        Ns, M = self.Ns, self.M
        N = Ns * Ns
        q = np.asarray(q).reshape(-1)
        G1 = np.zeros((M, M), dtype)
        G2 = np.zeros((M, M), dtype)
        G1[:Ns, :Ns] = q[:N].reshape(Ns, Ns)
        G2[:Ns, :Ns] = q[N:].reshape(Ns, Ns)
        A = rfft2(G1)
        B = rfft2(G2)
        kxx = self.spectra["xx"].astype(dtype)
        kyy = self.spectra["yy"].astype(dtype)
        kxy = self.spectra["xy"].astype(dtype)
        U = kxx * A + kxy * B
        V = kxy * A + kyy * B
        ux = irfft2(U, (M, M))[:Ns, :Ns]
        uy = irfft2(V, (M, M))[:Ns, :Ns]
        return np.concatenate([ux.reshape(-1), uy.reshape(-1)]).astype(dtype)
