"""Manufactured KKT optima and independent diagnostics for the certification
tests (restating the reference's tests/contact_oracle.hpp:35-60,147-158 and
tests/test_certification.cpp:34-46,76-148 on the FFT operators).

Given p* >= 0 and g* >= 0 with complementary support and a level alpha*,
g0 = alpha* 1 - S p* + g* makes (p*, alpha*) satisfy the KKT conditions of
min 1/2 p'Sp + p'g0, p >= 0, sum p = sum p* exactly: v = S p* + g0 =
alpha* + g*, so v - alpha* = g* >= 0 and p*_i g*_i = 0.  The reference
builds them on a small dense SPD matrix; here S is the fft / periodic
operator itself (the GPU path has no dense operator), applied in FP64 by
the CPU oracle.
"""

import numpy as np


def cases(Ns):
    """(name, p*, g*) on an Ns x Ns grid: a singleton support, full contact,
    and two islands with one degenerate p* = g* = 0 cell (the reference's
    three T01 cases, spread over the grid)."""
    N = Ns * Ns
    i = np.arange(N)
    out = []
    p = np.zeros(N)
    c = (Ns // 2) * Ns + Ns // 2
    p[c] = 1.0
    g = 0.5 + 0.1 * (i % 10)
    g[c] = 0.0
    out.append(("singleton", p, g))
    p = 0.3 + 0.05 * (i % 10)
    out.append(("full", p, np.zeros(N)))
    p = np.zeros(N)
    iy, ix = np.divmod(i, Ns)
    isl1 = (np.abs(iy - Ns // 4) <= 1) & (np.abs(ix - Ns // 4) <= 2)
    isl2 = (np.abs(iy - 3 * Ns // 4) <= 2) & (np.abs(ix - 2 * Ns // 3) <= 1)
    p[isl1] = 0.7 - 0.05 * (ix[isl1] - Ns // 4) ** 2
    p[isl2] = 0.4 + 0.1 * (iy[isl2] - 3 * Ns // 4)
    p[isl2] = np.maximum(p[isl2], 0.05)
    g = np.where(p > 0, 0.0, 0.3 + 0.2 * (i % 7) / 7.0)
    degen = (Ns // 2) * Ns + 3
    g[degen] = 0.0  # p* = g* = 0 there
    out.append(("islands+degenerate", p, g))
    return out


def manufacture(matvec, p_star, g_star, alpha_star=0.25):
    """tests/contact_oracle.hpp:147-158: g0 = alpha* - S p* + g*; returns
    (g0, P_total)."""
    g0 = alpha_star - matvec(p_star) + g_star
    return g0, float(p_star.sum())


def g_range(g0):
    r = float(np.max(g0) - np.min(g0))
    return r if r > 0.0 else 1.0


def diagnose(matvec, g0, p, P_total, g_ref):
    """tests/contact_oracle.hpp:35-60: every acceptance quantity recomputed
    from the returned pressure with separate arithmetic."""
    p = np.ravel(p)
    v = matvec(p) + g0
    on = p > 0.0
    nc = int(on.sum())
    approach = float(v[on].sum() / nc) if nc else float(v.min())
    vmin = float(v.min())
    G = float(np.sum(p * (v - vmin)))
    pk = float(np.sum(p * np.abs(v - approach)))
    return dict(approach=approach, min_gap=vmin - approach, fw_gap=G,
                fw_error=G / (P_total * g_ref),
                penetration=max(0.0, -(vmin - approach)) / g_ref,
                load_error=abs(float(p.sum()) - P_total) / P_total,
                min_pressure=float(p.min()), pk_error=pk / (P_total * g_ref), n_contact=nc)


def diagnostics_agree(r, d, atol):
    """tests/test_certification.cpp:34-46."""
    s = max(1.0, abs(d["fw_error"]))
    return (abs(r.fw_error - d["fw_error"]) <= atol * s
            and abs(r.penetration_error - d["penetration"]) <= atol
            and abs(r.load_error - d["load_error"]) <= atol
            and abs(r.approach - d["approach"]) <= atol * max(1.0, abs(d["approach"]))
            and abs(r.pk_error - d["pk_error"]) <= atol * max(1.0, d["pk_error"]))
