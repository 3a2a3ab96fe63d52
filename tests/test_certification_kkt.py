"""Manufactured KKT optimum (the reference's tests/test_certification.cpp:
76-148, T01) on the fft and periodic operators, CPU: the numpy oracle and
the reference's own C++ (oracle/_ref) both recover p* with certificates at
the 1e-12 level, an already optimal warm start takes 0 iterations and an
invalid one does not.  The GPU version is in test_gpu_configs.py."""

import numpy as np
import pytest

import manufactured as mf
from oracle import ref
from oracle.operators import FFTOperator, PeriodicFFTOperator
from oracle.solver import SolveOptions, SolveScales, solve_contact_impl

NS = 16


def _op(backend):
    return FFTOperator(NS) if backend == "fft" else PeriodicFFTOperator(NS)


def _check(r, p_star, g0, P, gref, mv, warm):
    d = mf.diagnose(mv, g0, r.pressure, P, gref)
    relp = np.linalg.norm(np.ravel(r.pressure) - p_star) / np.linalg.norm(p_star)
    assert r.status == "converged", (r.status, r.status_reason)
    assert d["min_pressure"] >= 0.0
    assert d["fw_error"] <= 1e-12 and d["penetration"] <= 1e-12 and d["load_error"] <= 1e-12
    assert mf.diagnostics_agree(r, d, 1e-9)
    assert relp < 1e-7, relp
    if warm == 1:
        assert r.iterations == 0
    if warm == 2:
        assert r.iterations > 0


def _warm(warm, p_star, P):
    if warm == 0:
        return None
    if warm == 1:
        return p_star.copy()
    p0 = np.zeros_like(p_star)
    p0[-1] = P
    return p0


@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("case", [0, 1, 2])
def test_manufactured_kkt_oracle(backend, case):
    op = _op(backend)
    mv = lambda x: op.matvec(x, np.float64)  # noqa: E731
    _, p_star, g_star = mf.cases(NS)[case]
    g0, P = mf.manufacture(mv, p_star, g_star)
    gref = mf.g_range(g0)
    opt = SolveOptions(tol=1e-12, max_iter=20000, scales=SolveScales(g_ref=gref))
    for warm in range(3):
        r = solve_contact_impl(mv, g0, P / g0.size, opt, None, _warm(warm, p_star, P),
                               dtype=np.float64)
        _check(r, p_star, g0, P, gref, mv, warm)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("case", [0, 1, 2])
def test_manufactured_kkt_reference(backend, case):
    s = ref.ContactSolver(NS, backend=backend)
    mv = lambda x: s.matvec(x)  # noqa: E731
    _, p_star, g_star = mf.cases(NS)[case]
    g0, P = mf.manufacture(mv, p_star, g_star)
    gref = mf.g_range(g0)
    for warm in range(3):
        r = s.solve(g0, P / g0.size, tol=1e-12, max_iter=20000, g_ref=gref,
                    p_init=_warm(warm, p_star, P))
        _check(r, p_star, g0, P, gref, mv, warm)
