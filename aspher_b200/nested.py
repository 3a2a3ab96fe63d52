"""``solve_nested`` for the fft / periodic backends (python/bindings.cpp:836-879).

The level loop, restriction / prolongation and precision staging run in the
library (``aspher_solve_nested``, the reference's solve_contact_nested,
src/nested_solve.cpp:518-990); this wrapper maps the reference's keyword
arguments onto ``aspher_nested_opts`` and returns a ``ContactResult``.
"""

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .api import ContactResult, _dev, _ptr, _stream, _to_device_f64

_ENGINE = {"auto": 0, "stencil": 1, "fft": 2}
_PRECISION = {"": 0, "double": 1, "float": 2, "float_then_double": 3}


def stencil_for_level(engine, precond, prev_occupancy, occupancy_max):
    """nested_solve.hpp:132-133 decision table."""
    return bool(L.lib().aspher_stencil_for_level(_ENGINE[engine], int(bool(precond)),
                                                 float(prev_occupancy), float(occupancy_max)))


def solve_nested(grid_size, gap, p_nominal, domain_size=1.0, E_star=1.0, coarsest=64, q=6,
                 leaf_side=8, precond=True, precond_engine="auto", precond_radius=2,
                 precond_occupancy_max=0.4, precond_cost_gate=0.0, tol=1e-8, coarse_tol=1e-4,
                 max_iter=20000, use_pr=True, single_precision=False, precision="",
                 float_floor=2e-6, allow_tolerance_relaxation=False, light_result=False,
                 backend="h2", record_error_history=False, active_set=False,
                 active_delta=0.05, active_halo=2, active_max_rounds=5,
                 active_all_levels=True, active_occupancy_max=0.4):
    """Single-entry nested-grid (cascadic) contact solve on the device.

    Same signature and defaults as the reference.  backend must be 'fft' or
    'periodic' (the reference default 'h2' is not part of this build).  The
    precond_cost_gate (opt-in, default off in the reference) is not
    implemented: a positive value raises ValueError.
    """
    if backend not in ("fft", "periodic"):
        raise ValueError("solve_contact_nested: backend must be 'fft' or 'periodic' on this "
                         "build (got %r)" % backend)
    if precond_engine not in _ENGINE:
        raise ValueError("precond_engine must be 'auto', 'stencil' or 'fft'")
    if precision not in _PRECISION:
        raise ValueError("precision must be 'double', 'float', 'float_then_double' or '' "
                         "(defer to single_precision)")
    if precond_cost_gate and precond_cost_gate > 0.0:
        raise ValueError("precond_cost_gate > 0 is not supported by this build")
    o = L.NestedOpts()
    L.lib().aspher_nested_opts_default(C.byref(o))
    o.tol = float(tol)
    o.max_iter = int(max_iter)
    o.use_pr = int(bool(use_pr))
    o.coarsest = int(coarsest)
    o.q = int(q)
    o.leaf_side = int(leaf_side)
    o.precond = int(bool(precond))
    o.precond_engine = _ENGINE[precond_engine]
    o.precond_radius = int(precond_radius)
    o.precond_occupancy_max = float(precond_occupancy_max)
    o.coarse_tol = float(coarse_tol)
    o.single_precision = int(bool(single_precision))
    o.precision = _PRECISION[precision]
    o.float_floor = float(float_floor)
    o.allow_tolerance_relaxation = int(bool(allow_tolerance_relaxation))
    o.light_result = int(bool(light_result))
    o.record_error_history = int(bool(record_error_history))
    o.active_set = int(bool(active_set))
    o.active_delta = float(active_delta)
    o.active_halo = int(active_halo)
    o.active_max_rounds = int(active_max_rounds)
    o.active_all_levels = int(bool(active_all_levels))
    o.active_occupancy_max = float(active_occupancy_max)
    Ns = int(grid_size)
    N = Ns * Ns
    dev = _dev()
    g0 = _to_device_f64(gap, N, dev)
    p = torch.empty(N, dtype=torch.float64, device=dev)
    u = g = None
    if not light_result:
        u = torch.empty(N, dtype=torch.float64, device=dev)
        g = torch.empty(N, dtype=torch.float64, device=dev)
    hcap = int(max_iter) + 1 if record_error_history else 0
    hist = np.zeros(max(hcap, 1), dtype=np.float64)
    stages = (L.Stage * 64)()
    nst = C.c_int(0)
    res = L.Result()
    L.check(L.lib().aspher_solve_nested(
        L.BACKEND[backend], Ns, float(domain_size), float(E_star), _ptr(g0), float(p_nominal),
        C.byref(o), _ptr(p), _ptr(u), _ptr(g),
        hist.ctypes.data_as(C.c_void_p) if hcap else C.c_void_p(0), hcap, C.byref(res),
        stages, 64, C.byref(nst), _stream()))
    r = ContactResult(res, Ns, p, u, g, hist[:res.history_len].copy() if hcap else None)
    r.stage_stats = [dict(name=st.name.decode(), precision=st.precision.decode(), q=st.q,
                          requested_tol=st.requested_tol, effective_tol=st.effective_tol,
                          iterations=st.iterations, matvec_count=st.matvec_count,
                          seconds=st.seconds, status=L.STATUS_NAMES[st.status],
                          fw_error=st.fw_error, penetration_error=st.penetration_error,
                          precond_dropped=bool(st.precond_dropped))
                     for st in stages[:nst.value]]
    r.time_build = res.time_build
    r.time_coarse = res.time_coarse
    r.time_candidate = res.time_candidate
    r.active_rounds = res.active_rounds
    r.active_fallback = bool(res.active_fallback)
    return r
