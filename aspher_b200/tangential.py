"""Tangential (Cerruti) FFT operator and the tangential projected CG on the device.

Mirrors the reference's ``TangentialFFTOperator`` over ``CerrutiKernel``
(include/tangential_operator.hpp:32-57, include/cerruti_kernel.hpp:35-61):
u = C q with q = [q_x; q_y] and u = [u_x; u_y] stacked, N = Ns^2 values
each in natural flat order, the dense block [[XX, XY], [XY, YY]] applied
exactly through the zero-padded (2Ns)^2 FFT.  ``solve`` is the
reference's ``solve_tangential`` (include/friction_solve.hpp:62-76) on it:
the vector Polonsky-Keer iteration under |q_i| <= s_i, displacement or
force control, with the local KKT check of the returned state.  The C ABI
is ``aspher_tan_create`` / ``aspher_tan_matvec`` / ``aspher_solve_tangential``
(include/aspher_b200.h).
"""

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .api import _dev, _ptr, _stream


class TangentialOperator:
    """TangentialFFTOperator(CerrutiKernel(grid_size, domain_size, E_star, nu))."""

    def __init__(self, grid_size, domain_size=1.0, E_star=1.0, nu=0.3):
        _dev()
        self.Ns = int(grid_size)
        self.N = self.Ns * self.Ns
        self.domain_size, self.E_star, self.nu = float(domain_size), float(E_star), float(nu)
        h = C.c_void_p()
        L.check(L.lib().aspher_tan_create(self.Ns, self.domain_size, self.E_star, self.nu,
                                          C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().aspher_tan_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def max_im_ratio(self):
        v = C.c_double()
        L.check(L.lib().aspher_tan_max_im_ratio(self._h, C.byref(v)))
        return v.value

    def matvec_(self, q, u):
        """u = C q on device tensors of 2 Ns^2 float32 or float64 values (may alias)."""
        if q.dtype not in (torch.float32, torch.float64) or u.dtype != q.dtype:
            raise ValueError("matvec: float32/float64 tensors of one dtype expected")
        if q.numel() != 2 * self.N or u.numel() != 2 * self.N:
            raise ValueError("matvec: q and u hold 2 Ns^2 values ([q_x; q_y])")
        if not (q.is_contiguous() and u.is_contiguous()):
            raise ValueError("matvec: contiguous tensors expected")
        dt = L.F64 if q.dtype == torch.float64 else L.F32
        L.check(L.lib().aspher_tan_matvec(self._h, dt, _ptr(q), _ptr(u), _stream()))
        return u

    def matvec(self, q):
        """u = C q for a float64 array of 2 Ns^2 values; returns a numpy array."""
        q = np.ascontiguousarray(np.asarray(q, np.float64).reshape(-1))
        if q.size != 2 * self.N:
            raise ValueError("matvec: q size != 2*Ns*Ns")
        x = torch.from_numpy(q).to(_dev())
        y = torch.empty_like(x)
        self.matvec_(x, y)
        return y.cpu().numpy()

    def tables(self):
        """(xx, yy, xy) signed offset tables, each [dy + Ns - 1, dx + Ns - 1]."""
        W = 2 * self.Ns - 1
        out = [np.empty(W * W) for _ in range(3)]
        L.check(L.lib().aspher_tan_tables(self._h, *[o.ctypes.data for o in out]))
        return tuple(o.reshape(W, W) for o in out)

    def solve(self, s, force_control=False, target=(0.0, 0.0), tol=1e-8, max_iter=5000,
              use_pr=True, kkt_tol=0.0, q_init=None, u_hist=None):
        """solve_tangential(C, s, force_control, target, tol, max_iter, use_pr)
        (unpreconditioned, FP64).  s: Ns^2 thresholds; target: the rigid
        shift (displacement control) or the mean traction (force control);
        q_init / u_hist: optional 2 Ns^2 warm start / history term.  Returns
        (q, result): q the stacked traction [q_x; q_y] as a numpy array and
        result a dict of the TangentialResult fields."""
        dev = _dev()

        def field(a, n, name):
            if a is None:
                return None
            t = torch.as_tensor(a, dtype=torch.float64).to(dev).reshape(-1).contiguous()
            if t.numel() != n:
                raise ValueError("%s has %d entries, expected %d" % (name, t.numel(), n))
            return t
        st = field(s, self.N, "s")
        q0 = field(q_init, 2 * self.N, "q_init")
        uh = field(u_hist, 2 * self.N, "u_hist")
        q = torch.empty(2 * self.N, dtype=torch.float64, device=dev)
        r = L.TanResult()
        L.check(L.lib().aspher_solve_tangential(
            self._h, _ptr(st), int(bool(force_control)), float(target[0]), float(target[1]),
            float(tol), int(max_iter), int(bool(use_pr)), float(kkt_tol), _ptr(q0), _ptr(uh),
            _ptr(q), C.byref(r), _stream()))
        out = {k: getattr(r, k) for k, _ in L.TanResult._fields_}
        out["status"] = L.STATUS_NAMES[r.status]
        out["status_reason"] = r.status_reason.decode()
        out["converged"] = bool(r.converged)
        out["delta_t"] = (r.delta_t[0], r.delta_t[1])
        out["q_mean"] = (r.q_mean[0], r.q_mean[1])
        return q.cpu().numpy(), out
