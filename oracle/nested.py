"""Nested-grid (cascadic) driver for the fft / periodic backends (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  Restates
``solve_contact_nested`` (src/nested_solve.cpp:518-990) without the H2
backend.  The active-set branch (``active_level``, nested_solve.cpp:72-518,
and the restricted PK ``solve_contact_active_impl``,
contact_solver.cpp:595-1040) is restated for the fft / periodic operators,
which the reference itself only pairs with h2 (nested_solve.cpp:608-617): the
restricted PK runs on the compressed candidate vectors, with the operator
and the preconditioner applied on the full grid and read back at the
candidates, and the full grid's load (``SolveOptions.n_grid``).
"""

import time

import numpy as np

from .operators import FFTOperator, PeriodicFFTOperator
from .precond import FourierPreconditioner, StencilPreconditioner
from .solver import SolveOptions, SolveScales, solve_contact_impl


def stencil_for_level(engine, precond, prev_occupancy, occupancy_max):
    """nested_solve.cpp:27-39."""
    if not precond:
        return False
    if engine == "stencil":
        return True
    if engine == "fft":
        return False
    return prev_occupancy < 0.0 or prev_occupancy < occupancy_max


def restrict_field(f, Ns):
    """2x2 block average, fine (Ns x Ns) -> coarse (nested_solve.cpp:42-54)."""
    a = np.asarray(f, dtype=np.float64).reshape(Ns, Ns)
    c = Ns // 2
    out = 0.25 * (((a[0::2, 0::2] + a[0::2, 1::2]) + a[1::2, 0::2]) + a[1::2, 1::2])
    return out.reshape(c * c)


def prolong_field(pc, Nc):
    """Injection, coarse -> fine (2Nc x 2Nc) (nested_solve.cpp:57-71)."""
    a = np.asarray(pc, dtype=np.float64).reshape(Nc, Nc)
    return np.repeat(np.repeat(a, 2, axis=0), 2, axis=1).reshape(-1)


def dilate_mask(m, Ns, r):
    """Chebyshev (square) dilation by r, clamped at the edges: a max filter
    along rows, then along columns (nested_solve.cpp:72-100)."""
    m = np.asarray(m, dtype=bool).reshape(Ns, Ns)
    if r <= 0:
        return m.reshape(-1).copy()
    tmp = np.zeros_like(m)
    for d in range(-r, r + 1):
        lo, hi = max(0, d), Ns + min(0, d)
        tmp[:, lo - d:hi - d] |= m[:, lo:hi]
    out = np.zeros_like(m)
    for d in range(-r, r + 1):
        lo, hi = max(0, d), Ns + min(0, d)
        out[lo - d:hi - d, :] |= tmp[lo:hi, :]
    return out.reshape(-1)


def active_level(op, pobj, glvl, p_bar, lvl_tol, max_iter, use_pr, n, p_init, coarse_gap,
                 g_ref, datum, dt, active_delta, active_halo, active_max_rounds,
                 record_history, light):
    """One restricted level (nested_solve.cpp:118-518): candidates from the
    coarse contact and gap, restricted PK at tol/2 on the compressed
    candidate vectors, the global check from a full-grid apply, dilated
    violations added per round, a full-grid fallback solve when no round
    certifies."""
    N = n * n
    R = np.dtype(dt).type
    gmax, gmin = float(np.max(glvl)), float(np.min(glvl))
    g_scale = gmax - gmin if gmax > gmin else 1.0
    delta = active_delta * g_scale
    vthresh = -lvl_tol * g_scale
    cm = dilate_mask(np.asarray(p_init) > 0.0, n, active_halo)
    cg = np.asarray(coarse_gap, dtype=np.float64).reshape(n // 2, n // 2)
    cm |= (np.repeat(np.repeat(cg, 2, axis=0), 2, axis=1) < delta).reshape(-1)
    g0c_full = (np.asarray(glvl, dtype=np.float64) - datum).astype(R)
    pw = np.asarray(p_init, dtype=np.float64)
    P_total = p_bar * N
    it_total, rounds, certified, res, hist = 0, 0, False, None, []
    while rounds < active_max_rounds:
        rounds += 1
        idx = np.nonzero(cm)[0]

        def S_c(x, idx=idx):
            xf = np.zeros(N, dtype=R)
            xf[idx] = x
            return op.matvec(xf, dt)[idx]

        pc = None
        if pobj is not None:
            def pc(g_, c_, idx=idx):
                gf = np.zeros(N, dtype=R)
                gf[idx] = g_
                cf = np.zeros(N, dtype=bool)
                cf[idx] = c_
                return pobj.apply(gf, cf, dt)[idx]

        aopt = SolveOptions(tol=0.5 * lvl_tol, requested_tol=lvl_tol, max_iter=max_iter,
                            use_pr=use_pr, record_history=record_history,
                            allow_tolerance_relaxation=True, n_grid=N,
                            scales=SolveScales(g_ref=g_ref, datum=datum, datum_mode="caller"))
        res = solve_contact_impl(S_c, g0c_full[idx], p_bar, aopt, pc, pw[idx], dtype=dt)
        it_total += res.iterations
        hist += list(res.error_history or [])
        pfull = np.zeros(N)
        pfull[idx] = res.pressure
        u = op.matvec(pfull.astype(R), dt).astype(np.float64)
        v = u + g0c_full.astype(np.float64)
        a = res.approach - datum
        vmin_glob = float(v.min())
        vmin_loc = float(v[idx].min())
        viol = (~cm) & (v - a < vthresh)
        G_glob = res.fw_gap + P_total * (vmin_loc - vmin_glob)
        fw_glob = G_glob / (P_total * g_ref)
        pen_glob = max(0.0, -(vmin_glob - a)) / g_ref
        res.fw_gap, res.fw_error, res.penetration_error = G_glob, fw_glob, pen_glob
        res.pressure = pfull
        res.gap = None if light else v - a
        if res.status == "converged" and not viol.any() and fw_glob <= lvl_tol \
                and pen_glob <= lvl_tol:
            certified = True
            break
        if not viol.any():
            break
        cm |= dilate_mask(viol, n, active_halo)
        pw = pfull
    fallback = False
    if not certified:
        fopt = SolveOptions(tol=lvl_tol, requested_tol=lvl_tol, max_iter=max_iter,
                            use_pr=use_pr, light=light, record_history=record_history,
                            keep_best=not light, allow_tolerance_relaxation=True,
                            scales=SolveScales(g_ref=g_ref, datum=datum, datum_mode="caller"))
        mv = (lambda x: op.matvec(x, dt))
        pcf = None if pobj is None else (lambda g_, c_: pobj.apply(g_, c_, dt))
        res = solve_contact_impl(mv, g0c_full, p_bar, fopt, pcf, res.pressure, dtype=dt)
        it_total += res.iterations
        hist += list(res.error_history or [])
        fallback = True
    res.iterations = it_total
    res.error_history = hist
    res.active_rounds = rounds
    res.active_fallback = fallback
    return res


def solve_contact_nested(Ns, L, E_star, g0, p_bar, tol=1e-8, max_iter=20000,
                         use_pr=True, coarsest=64, precond=True,
                         precond_engine="auto", precond_radius=2,
                         precond_occupancy_max=0.4, coarse_tol=1e-4,
                         single_precision=False, precision="",
                         float_floor=2e-6, allow_tolerance_relaxation=False,
                         light_result=False, backend="fft",
                         record_error_history=False, leaf_side=8, active_set=False,
                         active_delta=0.05, active_halo=2, active_max_rounds=5,
                         active_all_levels=True, active_occupancy_max=0.4, **_unused):
    g0 = np.asarray(g0, dtype=np.float64).reshape(-1)
    if Ns <= 0:
        raise ValueError("solve_contact_nested: Ns must be positive")
    if g0.size != Ns * Ns:
        raise ValueError("solve_contact_nested: g0 size != Ns*Ns")
    if not np.all(np.isfinite(g0)):
        raise ValueError("solve_contact_nested: gap contains non-finite values")
    if not (p_bar > 0.0):
        raise ValueError("solve_contact_nested: p_nominal must be positive")
    if not (tol > 0.0):
        raise ValueError("solve_contact_nested: tol must be positive")
    if coarsest <= 0 or coarsest > Ns:
        raise ValueError("solve_contact_nested: bad coarsest")
    if not (coarse_tol > 0.0):
        raise ValueError("solve_contact_nested: coarse_tol must be positive")
    if precision == "double" or (precision == "" and not single_precision):
        policy = "double"
    elif precision in ("float",) or (precision == "" and single_precision):
        policy = "float"
    elif precision == "float_then_double":
        policy = "float_then_double"
    else:
        raise ValueError("precision must be 'double', 'float', "
                         "'float_then_double' or ''")
    any_float = policy != "double"
    levels = []
    n = coarsest
    while n <= Ns:
        levels.append(n)
        n *= 2
    if not levels or levels[-1] != Ns:
        raise ValueError("solve_contact_nested: Ns must equal coarsest * 2^k")
    if backend not in ("fft", "periodic"):
        raise ValueError("oracle nested driver: backend must be fft or periodic")
    if active_set:
        if active_halo < 0 or active_max_rounds < 1 or not (active_delta >= 0.0) \
                or not (active_occupancy_max > 0.0):
            raise ValueError("solve_contact_nested: bad active-set parameters")
        if policy == "float_then_double":
            raise ValueError("solve_contact_nested: float_then_double with active_set")
        if len(levels) < 2:
            raise ValueError("solve_contact_nested: active_set needs a coarse level")

    ncoarse = len(levels) - 1
    gap = [None] * ncoarse
    if ncoarse > 0:
        gap[ncoarse - 1] = restrict_field(g0, Ns)
        for i in range(ncoarse - 2, -1, -1):
            gap[i] = restrict_field(gap[i + 1], levels[i + 1])
    g_min_f, g_max_f = float(g0.min()), float(g0.max())
    datum = g_min_f + 0.5 * (g_max_f - g_min_f)
    g_ref = max(g_max_f - g_min_f, p_bar * L / E_star)

    p_init = None
    coarse_gap = None
    prev_occupancy = -1.0
    stages = []
    res = None
    t0 = time.perf_counter()
    for li, n in enumerate(levels):
        if backend == "fft":
            op = FFTOperator(n, L, E_star)
        else:
            op = PeriodicFFTOperator(n, L, E_star)
        r_lvl = min(precond_radius, max(1, n // 4), leaf_side)
        engine = "fft" if (backend == "periodic" and precond_engine == "auto") \
            else precond_engine
        use_stencil = stencil_for_level(engine, precond, prev_occupancy,
                                        precond_occupancy_max)
        pobj = None
        if use_stencil:
            pobj = StencilPreconditioner(n, r_lvl)
        elif precond:
            pobj = FourierPreconditioner(n)
        finest = li + 1 == len(levels)
        glvl = g0 if finest else gap[li]
        polish_after = finest and policy == "float_then_double"
        lvl_tol = tol if finest else coarse_tol
        if polish_after:
            lvl_tol = float_floor
        elif any_float:
            lvl_tol = max(lvl_tol, float_floor)
        gate_open_next = prev_occupancy < 0.0 or prev_occupancy < active_occupancy_max
        keep_gap = bool(active_set and not finest and gate_open_next
                        and (active_all_levels or li + 2 == len(levels)))
        light = light_result if finest else not keep_gap
        use_active = bool(active_set and p_init is not None and coarse_gap is not None
                          and prev_occupancy < active_occupancy_max
                          and (finest or active_all_levels))
        opt = SolveOptions(tol=lvl_tol, requested_tol=(tol if finest else coarse_tol),
                           max_iter=max_iter, use_pr=use_pr, light=light,
                           record_history=finest and record_error_history,
                           keep_best=not light,
                           allow_tolerance_relaxation=(not finest) or polish_after
                           or allow_tolerance_relaxation,
                           scales=SolveScales(g_ref=g_ref, datum=datum,
                                              datum_mode="caller" if any_float
                                              else "solver"))
        if any_float:
            dt = np.float32
            gl = (glvl - datum).astype(np.float32)
        else:
            dt = np.float64
            gl = glvl
        mv = (lambda x, op=op, dt=dt: op.matvec(x, dt))
        pc = None
        if pobj is not None:
            pc = (lambda g_, c_, pobj=pobj, dt=dt: pobj.apply(g_, c_, dt))
        if use_active:
            res = active_level(op, pobj, glvl, p_bar, lvl_tol, max_iter, use_pr, n, p_init,
                               coarse_gap, g_ref, datum, dt, active_delta, active_halo,
                               active_max_rounds, finest and record_error_history, light)
        else:
            res = solve_contact_impl(mv, gl, p_bar, opt, pc, p_init, dtype=dt)
        coarse_gap = res.gap if keep_gap else None
        prev_occupancy = res.contact_fraction
        stages.append(dict(name=("finest:" if finest else "coarse:") + str(n)
                           + ("(active)" if use_active else ""),
                           precision="float" if any_float else "double",
                           requested_tol=opt.requested_tol, effective_tol=opt.tol,
                           iterations=res.iterations, matvec_count=res.matvec_count,
                           seconds=res.time_total, status=res.status,
                           fw_error=res.fw_error,
                           penetration_error=res.penetration_error))
        if polish_after:
            before = res
            popt = SolveOptions(tol=tol, requested_tol=tol, max_iter=max_iter,
                                use_pr=use_pr, light=light_result,
                                record_history=record_error_history,
                                keep_best=not light_result,
                                allow_tolerance_relaxation=allow_tolerance_relaxation,
                                scales=SolveScales(g_ref=g_ref, datum=datum,
                                                   datum_mode="solver"))
            mvd = (lambda x, op=op: op.matvec(x, np.float64))
            pcd = None
            if pobj is not None:
                pcd = (lambda g_, c_, pobj=pobj: pobj.apply(g_, c_, np.float64))
            res = solve_contact_impl(mvd, glvl, p_bar, popt, pcd, before.pressure,
                                     dtype=np.float64)
            stages.append(dict(name="polish:" + str(n), precision="double",
                               requested_tol=tol, effective_tol=tol,
                               iterations=res.iterations,
                               matvec_count=res.matvec_count,
                               seconds=res.time_total, status=res.status,
                               fw_error=res.fw_error,
                               penetration_error=res.penetration_error))
            res.iterations += before.iterations
            res.matvec_count += before.matvec_count
            res.precond_count += before.precond_count
            if record_error_history:
                res.error_history = before.error_history + res.error_history
        if not finest:
            p_init = prolong_field(res.pressure, n)
    res.stage_stats = stages
    res.time_total = time.perf_counter() - t0
    return res
