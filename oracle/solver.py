"""Polonsky-Keer projected CG with certified termination (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  A numpy restatement
of ``solve_contact_impl<Real>`` (src/contact_solver.cpp:150-587), of
``project_load_simplex`` (:31-60) and of the identification step (:314-364).
``dtype`` plays the role of ``Real``: vectors are kept in that precision and
every reduction is accumulated in float64, as in the reference.  Reduction
order differs from the reference's OpenMP partial sums, so results agree to
roundoff, not bit for bit (the reference's own tests state the same about
OpenMP reduction order, tests/test_fft.cpp:89-95).
"""

import math
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

STATUS_NAMES = ("converged", "stagnated", "max_iterations",
                "nonpositive_curvature", "nonfinite", "verification_failed",
                "resource_limit")  # contact_solver.hpp:13-21, .cpp:12-23


@dataclass
class SolveScales:
    """contact_solver.hpp:134-147."""
    p_ref: float = 0.0
    g_ref: float = 0.0
    datum_mode: str = "automatic"  # automatic | solver | caller
    datum: float = 0.0


@dataclass
class SolveOptions:
    """contact_solver.hpp:151-191."""
    tol: float = 1e-8
    requested_tol: float = 0.0
    max_iter: int = 5000
    use_pr: bool = True
    light: bool = False
    record_history: bool = False
    keep_best: bool = True
    load_tol: float = 0.0
    stall_limit: int = 200
    precond_cost_gate: float = 0.0
    allow_tolerance_relaxation: bool = False
    n_grid: int = 0  # > 0: the full grid's size when g0 holds a candidate subset
    scales: SolveScales = field(default_factory=SolveScales)


@dataclass
class ContactResult:
    """The fields of contact_solver.hpp:25-123 that this path fills."""
    pressure: np.ndarray = None
    displacement: Optional[np.ndarray] = None
    gap: Optional[np.ndarray] = None
    approach: float = 0.0
    objective: float = 0.0
    error: float = 0.0
    iterations: int = 0
    converged: bool = False
    contact_fraction: float = 0.0
    mean_pressure: float = 0.0
    error_history: List[float] = field(default_factory=list)
    status: str = "max_iterations"
    status_reason: str = ""
    pk_error: float = 0.0
    fw_gap: float = 0.0
    fw_error: float = 0.0
    load_error: float = 0.0
    pressure_violation: float = 0.0
    penetration_error: float = 0.0
    requested_tol: float = 0.0
    effective_tol: float = 0.0
    p_ref: float = 0.0
    g_ref: float = 0.0
    matvec_count: int = 0
    precond_count: int = 0
    identification_steps: int = 0
    returned_best: bool = False
    precond_dropped: bool = False
    time_total: float = 0.0
    time_matvec: float = 0.0
    time_precond: float = 0.0
    stage_stats: list = field(default_factory=list)

    @property
    def contact_area(self):
        return self.contact_fraction


def project_load_simplex(y, P_total):
    """In place p = max(y - theta, 0) with sum p = P (Michelot), returns theta.

    contact_solver.cpp:31-60; comparisons are double(y) > theta.
    """
    N = y.size
    if N == 0:
        return 0.0
    yd = y.astype(np.float64)
    ssum = float(np.sum(yd))
    nact = N
    theta = (ssum - P_total) / float(nact)
    for _ in range(64):
        sel = yd > theta
        n2 = int(np.count_nonzero(sel))
        s2 = float(np.sum(yd[sel]))
        if n2 == 0:
            break
        if n2 == nact:
            break
        nact = n2
        ssum = s2
        theta = (ssum - P_total) / float(nact)
    th = y.dtype.type(theta)
    y[...] = np.where(y > th, y - th, y.dtype.type(0))
    return theta


def _dsum(a):
    return float(np.sum(a, dtype=np.float64))


def solve_contact_impl(S: Callable, g0, p_bar, opt: SolveOptions,
                       precond: Optional[Callable] = None, p_init=None,
                       dtype=np.float64):
    """Polonsky & Keer projected CG (contact_solver.cpp:150-587).

    S(x) -> S x in ``dtype``; precond(g, contact_bool) -> z in ``dtype``.
    """
    R = np.dtype(dtype).type
    is_double = R is np.float64
    g0 = np.asarray(g0).astype(R, copy=False).reshape(-1)
    N = g0.size
    p_bar = R(p_bar)
    if N == 0 or not (p_bar > 0):
        raise ValueError("solve_contact: empty gap or p_bar <= 0")
    if not (opt.tol > 0.0):
        raise ValueError("solve_contact: tol must be positive")
    if opt.max_iter < 0:
        raise ValueError("solve_contact: max_iter must be >= 0")
    if not np.all(np.isfinite(g0)):
        raise ValueError("solve_contact: g0 contains non-finite values")

    # restricted solves see the candidate subset but carry the full grid's
    # load (contact_solver.cpp:628-630)
    N_grid = opt.n_grid if opt.n_grid > 0 else N
    P_total = float(p_bar) * N_grid
    gmin_v = float(g0.min())
    gmax_v = float(g0.max())
    g_ref = opt.scales.g_ref
    if not (g_ref > 0.0):
        g_ref = gmax_v - gmin_v
    if not (g_ref > 0.0):
        g_ref = 1.0
    p_ref = opt.scales.p_ref if opt.scales.p_ref > 0.0 else float(p_bar)
    load_tol = opt.load_tol if opt.load_tol > 0.0 else (1e-12 if is_double else 5e-7)
    tol = opt.tol
    req_tol = opt.requested_tol if opt.requested_tol > 0.0 else tol
    mode = opt.scales.datum_mode
    if mode == "automatic":
        datum = gmin_v + 0.5 * (gmax_v - gmin_v)
        subtract = True
    elif mode == "solver":
        datum = opt.scales.datum
        subtract = True
    else:
        datum = opt.scales.datum
        subtract = False
    gshift = R(datum) if subtract else R(0)
    # uniform start: p_bar, or P_total / Nc on a candidate subset
    p_unif = p_bar if N_grid == N else R(P_total / N)
    g0s = (g0 - gshift).astype(R)  # the Real expression g0(i) - gshift

    if p_init is not None:
        p = np.asarray(p_init).astype(R).reshape(-1).copy()
        if p.size != N:
            raise ValueError("solve_contact: p_init size mismatch")
        p = np.maximum(p, R(0))
        s = _dsum(p)
        if s > 0.0:
            p = (p * R(P_total / s)).astype(R)
        else:
            p = np.full(N, p_unif, dtype=R)
    else:
        p = np.full(N, p_unif, dtype=R)
    t = np.zeros(N, dtype=R)
    u = np.zeros(N, dtype=R)
    g = np.zeros(N, dtype=R)
    g_prev = np.zeros(N, dtype=R)
    best_p = None

    res = ContactResult()
    counters = {"mv": 0, "pc": 0, "t_mv": 0.0, "t_pc": 0.0}
    t_start = time.perf_counter()

    def apply(x):
        t0 = time.perf_counter()
        y = np.asarray(S(x)).astype(R, copy=False).reshape(-1)
        counters["t_mv"] += time.perf_counter() - t0
        counters["mv"] += 1
        return y

    def apply_precond(gin, mask):
        t0 = time.perf_counter()
        z = np.asarray(precond(gin, mask)).astype(R, copy=False).reshape(-1)
        counters["t_pc"] += time.perf_counter() - t0
        counters["pc"] += 1
        return z

    st = {"G_old": 1.0, "delta": R(0), "s_id": 0.0, "u_fresh": False}

    def evaluate():
        nonlocal g
        d = {}
        v = (u + g0s).astype(R)
        pos = p > 0
        vd = v.astype(np.float64)
        gsum = float(np.sum(vd[pos]))
        nc = int(np.count_nonzero(pos))
        vmin = float(vd.min()) if N else math.inf
        d["nc"] = nc
        alpha = gsum / nc if nc else vmin
        gmin = vmin - alpha
        a_R, gm_R = R(alpha), R(gmin)
        pd = p.astype(np.float64)
        pv = float(np.dot(pd, vd))
        g = (v - a_R).astype(R)
        gd = g.astype(np.float64)
        gcs = float(np.sum(gd[pos]))
        e = float(np.dot(pd, np.abs(gd)))
        Gc = float(np.dot(pd, (g - gm_R).astype(R).astype(np.float64)))
        psum = float(np.sum(pd))
        if nc > 0:  # refine_contact_mean, contact_solver.cpp:94-99
            delta = gcs / nc
            alpha += delta
            gmin -= delta
        d["alpha"], d["gmin"] = alpha, gmin
        d["pk"] = e / (P_total * g_ref)
        d["G"] = Gc
        d["fw"] = Gc / (P_total * g_ref)
        d["pen"] = max(0.0, -gmin) / g_ref
        d["psum"] = psum
        d["pv"] = pv
        d["load"] = abs(psum - P_total) / P_total
        d["finite"] = all(math.isfinite(x) for x in (gsum, vmin, psum, e, Gc))
        return d

    def identification_step():
        nonlocal p, u, t, g_prev
        pd = p.astype(np.float64)
        f_cur = float(np.dot(pd, 0.5 * u.astype(np.float64) + g0s.astype(np.float64)))
        if not (st["s_id"] > 0.0):
            pp = float(np.dot(pd, pd))
            pu = float(np.dot(pd, u.astype(np.float64)))
            st["s_id"] = pp / pu if (pu > 0.0 and pp > 0.0) else 1.0
        for trial in range(12):
            s = R(st["s_id"])
            z = (p - s * g).astype(R)
            project_load_simplex(z, P_total)
            r = apply(z)
            zd = z.astype(np.float64)
            f_try = float(np.dot(zd, 0.5 * r.astype(np.float64) + g0s.astype(np.float64)))
            gd = float(np.dot(g.astype(np.float64), (z - p).astype(R).astype(np.float64)))
            if math.isfinite(f_try) and gd < 0.0 and f_try <= f_cur + 1e-4 * gd:
                p, u = z, r
                st["u_fresh"] = True
                st["delta"] = R(0)
                t = np.zeros(N, dtype=R)
                g_prev = np.zeros(N, dtype=R)
                st["G_old"] = 1.0
                res.identification_steps += 1
                if trial == 0:
                    st["s_id"] *= 2.0
                return True
            st["s_id"] *= 0.25
        return False

    status = "max_iterations"
    reason = ""
    best_merit = math.inf
    seen_merit = math.inf
    stall = 0
    forced_id = 0
    stall_limit = opt.stall_limit if opt.stall_limit > 0 else 200
    d = None
    precond_on = precond is not None

    it = 0
    while it < opt.max_iter:
        if not st["u_fresh"]:
            u = apply(p)
        st["u_fresh"] = False
        d = evaluate()
        if not d["finite"]:
            status = "nonfinite"
            break
        if opt.record_history:
            res.error_history.append(d["pk"])
        if d["load"] <= load_tol and d["fw"] <= tol and d["pen"] <= tol:
            status = "converged"
            st["u_fresh"] = True
            break
        merit = max(d["fw"], d["pen"])
        if opt.keep_best and merit < best_merit:
            best_merit = merit
            best_p = p.copy()
        if merit < seen_merit * (1.0 - 1e-4):
            seen_merit = merit
            stall = 0
        else:
            stall += 1
            if stall >= stall_limit:
                if forced_id < 3 and identification_step():
                    forced_id += 1
                    stall = 0
                    it += 1
                    continue
                status = "stagnated"
                reason = "stall"
                break

        did_cg = False
        if d["nc"] >= 2:
            contact = p > 0
            if precond_on:
                z = apply_precond(g, contact)
            else:
                z = np.where(contact, g, R(0)).astype(R)
            zc = z[contact].astype(np.float64)
            gc_ = g[contact].astype(np.float64)
            G = float(np.dot(zc, gc_))
            G_pr = float(np.dot(zc, (g - g_prev).astype(R)[contact].astype(np.float64)))
            gg = float(np.dot(gc_, gc_))
            G_old = st["G_old"]
            if G_old != 0.0:
                beta_val = max(0.0, G_pr / G_old) if opt.use_pr else G / G_old
            else:
                beta_val = 0.0
            beta = R(st["delta"] * R(beta_val))
            t = np.where(contact, (z + beta * t).astype(R), R(0)).astype(R)
            g_prev = g.copy()
            st["G_old"] = G

            r = apply(t)
            rsum = _dsum(r[contact])
            num = float(np.dot(g[contact].astype(np.float64), t[contact].astype(np.float64)))
            rmean = R(rsum / d["nc"] if d["nc"] else 0.0)
            den = float(np.dot((r - rmean).astype(R)[contact].astype(np.float64),
                               t[contact].astype(np.float64)))
            if den > 0.0 and math.isfinite(den) and math.isfinite(num):
                tau = R(num / den)
                tau_ov = R(num * num / (den * gg)) if gg > 0.0 else tau
                was = p > 0
                pi = np.where(was, np.maximum((p - tau * t).astype(R), R(0)), p).astype(R)
                act = (pi == 0) & (g < 0)
                pi = np.where(act, (pi - tau_ov * g).astype(R), pi).astype(R)
                changed = bool(np.any((pi > 0) != was))
                p = pi
                st["delta"] = R(0) if changed else R(1)
                total = _dsum(p)
                if total > 0.0:
                    p = (p * R(P_total / total)).astype(R)
                else:
                    p = np.full(N, p_unif, dtype=R)
                did_cg = True
        if not did_cg:
            if not identification_step():
                status = "nonpositive_curvature"
                break
        it += 1

    if status != "converged" and opt.keep_best and best_p is not None:
        merit = max(d["fw"], d["pen"])
        if not (merit <= best_merit):
            p = best_p
            st["u_fresh"] = False
            res.returned_best = True
    if not st["u_fresh"]:
        u = apply(p)
    d = evaluate()
    if not d["finite"] and status != "nonfinite":
        status = "nonfinite"
    if status == "converged" and not (d["load"] <= load_tol and d["fw"] <= tol
                                      and d["pen"] <= tol):
        status = "verification_failed"
        reason = "final_check"
    if status == "converged" and req_tol < tol and not opt.allow_tolerance_relaxation:
        if not (d["fw"] <= req_tol and d["pen"] <= req_tol):
            status = "stagnated"
            reason = "precision_limit"

    if not opt.light:
        res.displacement = u.astype(np.float64)
        res.gap = g.astype(np.float64)
    res.approach = d["alpha"] + datum
    obj = float(np.dot(p.astype(np.float64),
                       0.5 * u.astype(np.float64) + g0s.astype(np.float64)))
    res.objective = obj + datum * P_total
    res.iterations = it
    res.contact_fraction = d["nc"] / N_grid
    res.mean_pressure = d["psum"] / N_grid
    res.status = status
    res.status_reason = reason
    res.converged = status == "converged"
    res.error = d["pk"]
    res.pk_error = d["pk"]
    res.fw_gap = d["G"]
    res.fw_error = d["fw"]
    res.load_error = d["load"]
    res.penetration_error = d["pen"]
    res.requested_tol = req_tol
    res.effective_tol = tol
    res.p_ref = p_ref
    res.g_ref = g_ref
    res.matvec_count = counters["mv"]
    res.precond_count = counters["pc"]
    res.time_matvec = counters["t_mv"]
    res.time_precond = counters["t_pc"]
    res.time_total = time.perf_counter() - t_start
    res.pressure = p.astype(np.float64)
    return res
