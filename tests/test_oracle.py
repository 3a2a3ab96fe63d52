"""Pins of the CPU oracle against the reference's golden values and gates.

These run without a GPU.  Each test names the reference test it restates.
"""

import os

import numpy as np
import pytest

from oracle.api import ContactSolver
from oracle.love import assemble_dense, boussinesq_table, love_uz
from oracle.operators import FFTOperator, PeriodicFFTOperator
from oracle.precond import FourierPreconditioner, StencilPreconditioner
from oracle.solver import SolveOptions, project_load_simplex, solve_contact_impl

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

# tests/test_stencil.cpp:21-33 (universal constants of w = F^-1|k| / w(0,0))
STENCIL_GOLDEN = {(0, 0): 1.0, (1, 0): -0.180875, (1, 1): -0.032860, (2, 0): 0.021189,
                  (2, 1): -0.003912, (2, 2): -0.003198}


def test_love_golden_fixture():
    d = np.loadtxt(os.path.join(GOLDEN, "love_golden.txt"))
    got = love_uz(d[:, 0], d[:, 1], d[:, 2], d[:, 3])
    assert np.all(np.isfinite(got)) and np.all(got > 0)
    rel = np.abs(got - d[:, 4]) / np.abs(d[:, 4])
    assert rel.max() <= 1e-12  # test_kernel_stability.cpp:53-83 gate


def test_love_reference_fixture():
    """The reference's own 80-digit fixture (tests/data/love_reference.txt,
    read by test_kernel_stability.cpp:53-83), committed as
    tests/golden/love_reference.txt by make_reference_fixtures_txt.py."""
    r = np.loadtxt(os.path.join(GOLDEN, "love_reference.txt"))
    assert len(r) == 472
    got = love_uz(r[:, 0], r[:, 1], r[:, 2], r[:, 3])
    rel = np.abs(got - r[:, 4]) / np.abs(r[:, 4])
    assert rel.max() <= 1e-12


def test_self_term_and_decay():
    """test_kernel.cpp:21-53."""
    Ns, L, E = 64, 1.0, 1.7
    h = L / Ns
    T = boussinesq_table(Ns, L, E)
    exact = 4.0 * h * np.log(1.0 + np.sqrt(2.0)) / (np.pi * E)
    assert abs(T[0, 0] / exact - 1.0) < 1e-14
    row = T[0, :]
    assert np.all(row > 0) and np.all(np.diff(row) < 0)

    def rel(dx, dy):
        r = h * np.hypot(dx, dy)
        return abs(T[dy, dx] / (h * h / (np.pi * E * r)) - 1.0)
    assert 0.03 < rel(1, 0) < 0.05 and 0.015 < rel(1, 1) < 0.035
    assert rel(5, 0) < 0.002 and rel(4, 3) < 0.002 and rel(20, 11) < 0.0005


@pytest.mark.parametrize("Ns", [24, 32, 64])
def test_fft_matvec_equals_dense(Ns):
    """test_fft.cpp:20-39: double < 1e-12, float < 1e-5."""
    S = assemble_dense(Ns, 1.0, 1.0)
    op = FFTOperator(Ns)
    x = np.random.default_rng(Ns).uniform(-1, 1, Ns * Ns)
    ref = S @ x
    assert np.linalg.norm(op.matvec(x) - ref) / np.linalg.norm(ref) < 1e-12
    yf = op.matvec(x.astype(np.float32), np.float32)
    assert np.linalg.norm(yf - ref) / np.linalg.norm(ref) < 1e-5


def test_periodic_modes_and_dc():
    """test_periodic.cpp:16-51."""
    n, L, Es = 32, 3.0, 2.5
    op = PeriodicFFTOperator(n, L, Es)
    ix = np.arange(n)
    for mx, my in ((1, 0), (0, 3), (2, 5)):
        q = 2 * np.pi * np.hypot(mx, my) / L
        ph = 2 * np.pi * (mx * ix[None, :] + my * ix[:, None]) / n
        p = np.cos(ph).ravel()
        u = op.matvec(p)
        ref = 2.0 / (Es * q) * p
        assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 2e-13
    assert np.linalg.norm(PeriodicFFTOperator(n).matvec(np.ones(n * n))) < 1e-13


def test_stencil_weights_golden():
    """test_stencil.cpp:37-55 (S1): 13 taps, 6 figures, centre exactly 1."""
    for Ns in (512, 1024, 2048):
        sp = StencilPreconditioner(Ns, 2)
        assert sp.ntaps() == 13
        for dx, dy, w in zip(sp.tap_dx, sp.tap_dy, sp.tap_w):
            a, b = abs(dx), abs(dy)
            key = (max(a, b), min(a, b))
            assert abs(w - STENCIL_GOLDEN[key]) <= 5e-6
            if dx == 0 and dy == 0:
                assert w == 1.0


def test_preconditioners_offset_blind_and_symmetric():
    """test_precond.cpp:27-66: Pi_C W Pi_C is symmetric and offset blind."""
    Ns = 32
    rng = np.random.default_rng(3)
    c = rng.random(Ns * Ns) < 0.4
    for P in (StencilPreconditioner(Ns, 2), FourierPreconditioner(Ns)):
        g = rng.standard_normal(Ns * Ns)
        z1 = P.apply(g, c, np.float64)
        z2 = P.apply(g + 123.456 * c, c, np.float64)
        assert np.linalg.norm(z1 - z2) <= 1e-12 * np.linalg.norm(z1)
        a = rng.standard_normal(Ns * Ns) * c
        b = rng.standard_normal(Ns * Ns) * c
        lhs = a @ P.apply(b, c, np.float64)
        rhs = b @ P.apply(a, c, np.float64)
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_hertz_fft_matches_dense():
    """test_fft.cpp:63-107: iterations +-1, same contact, pressure rel < 1e-6."""
    Ns, R, pbar = 64, 0.5, 0.05
    h = 1.0 / Ns
    x = (np.arange(Ns) + 0.5) * h - 0.5
    g0 = ((x[None, :] ** 2 + x[:, None] ** 2) / (2 * R)).ravel()
    rd = ContactSolver(Ns, backend="dense").solve(g0, pbar, 1e-8, 2000)
    rf = ContactSolver(Ns, backend="fft").solve(g0, pbar, 1e-8, 2000)
    assert rd.status == "converged" and rf.status == "converged"
    assert abs(rd.iterations - rf.iterations) <= 1
    assert rd.contact_fraction == rf.contact_fraction
    assert np.linalg.norm(rf.pressure - rd.pressure) / np.linalg.norm(rd.pressure) < 1e-6


def test_westergaard():
    """test_periodic.cpp:94-129."""
    n, L, Es, D = 256, 2.0, 1.3, 0.01
    pstar = np.pi * Es * D / L
    op = PeriodicFFTOperator(n, L, Es)
    cosx = np.tile(np.cos(2 * np.pi * np.arange(n) / n), (n, 1)).ravel()
    g0 = D * (1 - cosx)
    r = solve_contact_impl(op.matvec, g0, 1.5 * pstar, SolveOptions(tol=1e-12))
    assert r.status == "converged"
    pex = 1.5 * pstar + pstar * cosx
    assert np.linalg.norm(r.pressure - pex) / np.linalg.norm(pex) < 1e-9
    r = solve_contact_impl(op.matvec, g0, 0.3 * pstar, SolveOptions(tol=1e-10))
    assert r.status == "converged"
    width = (r.pressure[:n] > 0).sum() * L / n
    wex = 2 * (L / np.pi) * np.arcsin(np.sqrt(0.3))
    assert abs(width - wex) <= 2 * L / n


def test_simplex_projector_vs_sorting():
    """test_certification.cpp:443-467 (T21): Michelot == sorting projector."""
    rng = np.random.default_rng(21)
    for _ in range(200):
        n = int(rng.integers(1, 40))
        y = rng.standard_normal(n) * rng.uniform(0.1, 10)
        P = float(rng.uniform(0.1, 5.0))
        z = y.copy()
        project_load_simplex(z, P)
        u = np.sort(y)[::-1]
        css = np.cumsum(u) - P
        k = np.nonzero(u - css / np.arange(1, n + 1) > 0)[0][-1]
        ref = np.maximum(y - css[k] / (k + 1), 0)
        assert np.max(np.abs(z - ref)) <= 1e-12 * max(1.0, np.abs(y).max())
        assert abs(z.sum() - P) <= 1e-12 * max(P, 1.0)


def test_singleton_warm_start_repaired():
    """test_certification_py.py:42-73: an all-in-one-corner warm start is
    repaired to the cold solution."""
    ns = 8
    x = (np.arange(ns) + 0.5) / ns - 0.5
    g0 = (x[:, None] ** 2 + x[None, :] ** 2).ravel()
    op = ContactSolver(ns, backend="dense")
    warm = np.zeros(ns * ns)
    warm[0] = 0.01 * ns * ns
    cold = op.solve(g0, 0.01, tol=1e-10)
    got = op.solve(g0, 0.01, tol=1e-10, p_init=warm)
    assert got.status == "converged" and got.iterations > 0
    rel = np.linalg.norm(got.pressure - cold.pressure) / np.linalg.norm(cold.pressure)
    assert rel < 1e-6


def test_dilate_mask_chebyshev_clamped():
    """nested_solve.cpp:72-100: square (Chebyshev) dilation, clamped at the
    grid edges (no wrap)."""
    from oracle.nested import dilate_mask
    n = 9
    m = np.zeros(n * n, bool)
    m[0] = True            # corner (0, 0)
    m[4 * n + 6] = True    # (4, 6)
    d = dilate_mask(m, n, 2).reshape(n, n)
    ref = np.zeros((n, n), bool)
    ref[0:3, 0:3] = True
    ref[2:7, 4:9] = True
    assert np.array_equal(d, ref)
    assert np.array_equal(dilate_mask(m, n, 0), m)


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_oracle_active_set_nested_matches_full(backend):
    """The restricted (active-set) levels certify the full problem: the
    result equals the full nested solve within the tolerance; a candidate
    set without halo or gap margin needs an expansion round or the
    fallback, and still certifies."""
    from oracle.nested import solve_contact_nested
    from aspher_b200.surfaces import self_affine_gap
    ns, tol = 128, 1e-7
    g = self_affine_gap(ns, hurst=0.8, rms=0.002, seed=42)
    kw = dict(coarsest=32, tol=tol, backend=backend, light_result=True)
    full = solve_contact_nested(ns, 1.0, 1.0, g, 0.005, **kw)
    act = solve_contact_nested(ns, 1.0, 1.0, g, 0.005, active_set=True, **kw)
    assert full.status == "converged" and act.status == "converged"
    assert [s["name"] for s in act.stage_stats] == ["coarse:32", "coarse:64(active)",
                                                    "finest:128(active)"]
    assert act.fw_error <= tol and act.penetration_error <= tol
    rel = np.linalg.norm(act.pressure - full.pressure) / np.linalg.norm(full.pressure)
    assert rel <= 20 * tol
    tight = solve_contact_nested(ns, 1.0, 1.0, g, 0.005, active_set=True, active_halo=0,
                                 active_delta=0.0, active_max_rounds=1, **kw)
    assert tight.status == "converged" and tight.active_rounds == 1
    rel = np.linalg.norm(tight.pressure - full.pressure) / np.linalg.norm(full.pressure)
    assert rel <= 20 * tol
    # above active_occupancy_max (the coarse contact fraction) no level is restricted
    gated = solve_contact_nested(ns, 1.0, 1.0, g, 0.005, active_set=True,
                                 active_occupancy_max=1e-6, **kw)
    assert not any("(active)" in s["name"] for s in gated.stage_stats)
    with pytest.raises(ValueError):
        solve_contact_nested(ns, 1.0, 1.0, g, 0.005, active_set=True,
                             precision="float_then_double", **kw)
