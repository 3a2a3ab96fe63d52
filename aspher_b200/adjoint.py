"""Derivatives of the contact solve: the adjoint and a torch.autograd.Function.

No reference counterpart (the reference solve is not differentiable).  At a
converged solve with contact set C = {p > 0} the solution is locally the
solution of the equality-constrained system on C (S_CC p_C - alpha 1 = -g0_C,
sum_C p = P = p_bar N), so for a loss L(p) with w = dL/dp

    dL/dg0 = -lam (0 off C),   dL/dp_bar = -mu N,
    S_CC lam - mu 1 = w_C,     sum_C lam = 0,

which ``aspher_adjoint`` solves by CG on the contact set with the same
operator (and the stencil preconditioner).  Only the converged pressure is
kept from the forward solve; its iterates are never stored.
"""

import ctypes as C

import torch

from . import _lib as L
from .api import ContactSolver, Operator, solve_device, solve_device_mixed

_ADJ_PRECOND = {"none": 0, "": 0, "fourier": 1}


def adjoint(op, pressure, w, tol=1e-10, max_iter=5000, precond="fourier", radius=2,
            dtype=torch.float64):
    """(dL/dg0, dL/dp_bar, info) for the converged pressure of a solve on
    ``op`` and w = dL/dp (device tensors of N entries).  ``dtype`` is the
    working precision of the CG (FP64 reductions either way)."""
    if precond not in _ADJ_PRECOND:
        raise ValueError("adjoint precond must be 'none' or 'fourier'")
    N = op.N
    dev = pressure.device
    p = pressure.to(device=dev, dtype=torch.float64).contiguous().reshape(-1)
    wv = w.to(device=dev, dtype=torch.float64).contiguous().reshape(-1)
    if p.numel() != N or wv.numel() != N:
        raise ValueError("adjoint: pressure and w must have %d entries" % N)
    grad = torch.empty(N, dtype=torch.float64, device=dev)
    gp = C.c_double(0.0)
    info = L.AdjointInfo()
    L.check(L.lib().aspher_adjoint(
        op.handle, L.F64 if dtype == torch.float64 else L.F32, C.c_void_p(p.data_ptr()),
        C.c_void_p(wv.data_ptr()), C.c_double(tol), int(max_iter), _ADJ_PRECOND[precond],
        int(radius), C.c_void_p(grad.data_ptr()), C.byref(gp), C.byref(info),
        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    st = L.lib().aspher_status_string(info.status).decode()
    return grad, gp.value, dict(status=st, iterations=info.iterations,
                                contact_count=info.contact_count, residual=info.residual,
                                mu=info.mu, time=info.time)


class _ContactSolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, gap, p_nominal, op, cfg):
        g0 = gap.detach().to(torch.float64).contiguous().reshape(-1)
        pn = float(p_nominal)
        if cfg["precision"] == "double":
            r = solve_device(op, g0, pn, tol=cfg["tol"], max_iter=cfg["max_iter"],
                             precond=cfg["precond"], dtype=torch.float64, light=True)
        else:
            r, _ = solve_device_mixed(op, g0, pn, tol=cfg["tol"], max_iter=cfg["max_iter"],
                                      precond=cfg["precond"], light=True,
                                      polish=cfg["precision"] == "float_then_double")
        if r.status != "converged":
            raise RuntimeError("contact solve did not converge (%s); its derivative is "
                               "undefined" % r.status)
        p = r.pressure_device.reshape(-1)
        ctx.save_for_backward(p)
        ctx.op = op
        ctx.cfg = cfg
        ctx.gshape = gap.shape
        ctx.gdtype = gap.dtype
        ctx.pn_is_tensor = torch.is_tensor(p_nominal)
        return p.reshape(gap.shape).to(gap.dtype)

    @staticmethod
    def backward(ctx, grad_p):
        (p,) = ctx.saved_tensors
        cfg = ctx.cfg
        grad_g0, grad_pbar, info = adjoint(ctx.op, p, grad_p.reshape(-1),
                                           tol=cfg["adjoint_tol"],
                                           max_iter=cfg["adjoint_max_iter"],
                                           precond=cfg["adjoint_precond"],
                                           dtype=cfg["adjoint_dtype"])
        if info["status"] != "converged":
            raise RuntimeError("adjoint CG did not converge (%s)" % info["status"])
        gg = grad_g0.reshape(ctx.gshape).to(ctx.gdtype)
        gpn = (torch.tensor(grad_pbar, dtype=torch.float64, device=p.device)
               if ctx.pn_is_tensor else None)
        return gg, gpn, None, None


def contact_pressure(solver_or_op, gap, p_nominal, tol=1e-8, max_iter=5000, precond="fourier",
                     precision="double", adjoint_tol=1e-10, adjoint_max_iter=5000,
                     adjoint_precond="fourier", adjoint_dtype=torch.float64):
    """Differentiable contact pressure p(gap, p_nominal) on the device.

    ``solver_or_op``: a ContactSolver or an Operator.  ``gap`` a CUDA tensor
    of N (or Ns x Ns) entries, ``p_nominal`` a float or a 0-d tensor.  The
    forward pass is the product solve (``precision`` 'double', 'float' or
    'float_then_double'); backward runs the adjoint in ``adjoint_dtype``.
    """
    op = solver_or_op.op if isinstance(solver_or_op, ContactSolver) else solver_or_op
    if not isinstance(op, Operator):
        raise TypeError("contact_pressure needs a ContactSolver or an Operator")
    cfg = dict(tol=tol, max_iter=max_iter, precond=precond, precision=precision,
               adjoint_tol=adjoint_tol, adjoint_max_iter=adjoint_max_iter,
               adjoint_precond=adjoint_precond, adjoint_dtype=adjoint_dtype)
    return _ContactSolveFn.apply(gap, p_nominal, op, cfg)
