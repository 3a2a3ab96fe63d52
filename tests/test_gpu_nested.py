"""Nested-grid driver on the device vs single-level solves and the oracle.

Restates tests/test_periodic_py.py:54-102, tests/test_nested.py:15-90 and
tests/test_certification_py.py:75-121 of the reference for the fft /
periodic backends.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _rough(ns, seed=3, rms=0.01, k_hi=None):
    from aspher_b200 import self_affine_gap
    g = self_affine_gap(ns, hurst=0.8, rms=rms, k_lo=2.0, k_hi=k_hi or ns / 8, seed=seed)
    return g - g.min()


def rel(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_nested_matches_single_level_and_precisions():
    import aspher_b200 as hc
    ns, pbar = 256, 0.01
    g = _rough(ns)
    s = hc.ContactSolver(ns, domain_size=1.0, E_star=1.0, backend="periodic")
    ref = s.solve(g, pbar, tol=1e-12, precond="fourier-fft").pressure
    for prec, tol, bound in (("double", 1e-10, 1e-7), ("float_then_double", 1e-10, 1e-7),
                             ("float", 2e-6, 1e-4)):
        r = hc.solve_nested(grid_size=ns, gap=g, p_nominal=pbar, coarsest=32,
                            backend="periodic", tol=tol, precision=prec)
        assert r.status == "converged", (prec, r.status, r.status_reason)
        p = np.asarray(r.pressure).ravel()
        assert abs(p.mean() - pbar) < 1e-6 * pbar
        assert rel(p, ref) < bound, prec
        names = [st["name"] for st in r.stage_stats]
        assert names[0] == "coarse:32" and names[-1] in ("finest:256", "polish:256")


def test_auto_engine_is_fft_on_periodic():
    import aspher_b200 as hc
    ns = 256
    g = _rough(ns)
    runs = {e: hc.solve_nested(grid_size=ns, gap=g, p_nominal=0.02, coarsest=32,
                               backend="periodic", tol=1e-10, precond_engine=e)
            for e in ("auto", "fft", "stencil")}
    assert runs["auto"].iterations == runs["fft"].iterations
    assert runs["auto"].matvec_count == runs["fft"].matvec_count
    np.testing.assert_allclose(runs["auto"].pressure, runs["fft"].pressure, rtol=0, atol=1e-12)
    assert runs["stencil"].iterations > runs["fft"].iterations


def test_active_set_bad_arguments():
    """nested_solve.cpp:567-580,593-597,608-617: the active-set argument
    checks (the backend restriction to h2 excepted: this build restricts
    the fft / periodic levels)."""
    import aspher_b200 as hc
    g = _rough(128)
    for kw in (dict(precision="float_then_double"), dict(coarsest=128),
               dict(active_halo=-1), dict(active_max_rounds=0), dict(active_delta=-0.1),
               dict(active_occupancy_max=0.0)):
        args = dict(coarsest=32)
        args.update(kw)
        with pytest.raises(ValueError):
            hc.solve_nested(grid_size=128, gap=g, p_nominal=0.01, backend="periodic",
                            active_set=True, **args)
    with pytest.raises(ValueError):
        hc.solve_nested(grid_size=128, gap=g, p_nominal=0.01, coarsest=48, backend="fft")
    with pytest.raises(ValueError):
        hc.solve_nested(grid_size=128, gap=g, p_nominal=0.01, backend="h2")


def test_nested_fft_matches_oracle():
    import aspher_b200 as hc
    from oracle.api import solve_nested as osolve
    ns, pbar, tol = 256, 0.02, 1e-8
    g = _rough(ns, seed=7, rms=0.02, k_hi=16)
    r = hc.solve_nested(ns, g, pbar, coarsest=64, backend="fft", tol=tol)
    o = osolve(ns, g, pbar, coarsest=64, backend="fft", tol=tol)
    assert r.status == "converged" and o.status == "converged"
    assert rel(r.pressure, o.pressure) <= 10 * tol
    assert abs(r.contact_area - o.contact_area) <= 1e-4
    assert abs(r.iterations - o.iterations) <= max(2, o.iterations // 5)


def test_float_precision_policy():
    """test_nested.py:43-90: float-only asked for 1e-8 reports precision_limit,
    accepts the float floor when allowed, and float_then_double polishes."""
    import aspher_b200 as hc
    ns, pbar = 256, 0.05
    g = _rough(ns, seed=11)
    ref = hc.ContactSolver(ns, backend="fft").solve(g, pbar, tol=1e-8, precond="fourier")
    sp = hc.solve_nested(ns, g, pbar, coarsest=64, backend="fft", single_precision=True,
                         light_result=True)
    assert not sp.converged
    assert sp.status == "stagnated" and sp.status_reason == "precision_limit"
    assert sp.requested_tol < sp.effective_tol
    spr = hc.solve_nested(ns, g, pbar, coarsest=64, backend="fft", single_precision=True,
                          light_result=True, allow_tolerance_relaxation=True)
    assert spr.converged and spr.displacement is None
    assert rel(spr.pressure, ref.pressure) < 1e-3
    ftd = hc.solve_nested(ns, g, pbar, coarsest=64, backend="fft",
                          precision="float_then_double")
    assert ftd.status == "converged" and ftd.fw_error <= ftd.requested_tol
    assert rel(ftd.pressure, ref.pressure) < rel(spr.pressure, ref.pressure)
    assert ftd.stage_stats[-1]["name"].startswith("polish:")
    assert ftd.stage_stats[-2]["precision"] == "float"
    assert ftd.stage_stats[-1]["precision"] == "double"


def test_gap_datum_invariance_nested():
    """test_certification_py.py:92-121."""
    import aspher_b200 as hc
    ns, pbar = 128, 0.02
    g0 = _rough(ns, seed=7, rms=0.02, k_hi=16)
    ref = hc.solve_nested(ns, g0, pbar, coarsest=32, backend="fft", tol=1e-10)
    assert ref.status == "converged"
    for shift in (0.0, 1e3, 1e6):
        for single in (False, True):
            r = hc.solve_nested(ns, g0 + shift, pbar, coarsest=32, backend="fft",
                                single_precision=single, allow_tolerance_relaxation=single,
                                tol=1e-8)
            assert r.status == "converged"
            assert abs(r.approach - ref.approach - shift) < 1e-6 * max(1.0, shift)
            assert rel(r.pressure, ref.pressure) < (1e-4 if single else 1e-5)


@pytest.mark.parametrize("backend,precision", [("fft", "double"), ("fft", "float"),
                                               ("periodic", "double"), ("periodic", "float")])
def test_active_set_nested_matches_full_and_oracle(backend, precision):
    """Restricted (active-set) levels: a certified restricted solve is a
    certified solve of the full problem (global Frank-Wolfe gap and
    penetration from a full-grid apply), so it agrees with the full nested
    solve and with the oracle's restricted driver within the certified
    tolerance."""
    import aspher_b200 as hc
    from oracle.nested import solve_contact_nested as onested
    ns, pbar = 256, 0.005
    tol = 1e-7 if precision == "double" else 2e-6
    g = hc.self_affine_gap(ns, hurst=0.8, rms=0.002, seed=42)
    kw = dict(coarsest=64, tol=tol, precision=precision, backend=backend, light_result=False)
    full = hc.solve_nested(ns, g, pbar, **kw)
    act = hc.solve_nested(ns, g, pbar, active_set=True, **kw)
    ora = onested(ns, 1.0, 1.0, g, pbar, active_set=True, **kw)
    assert full.status == "converged" and act.status == "converged" and ora.status == "converged"
    names = [st["name"] for st in act.stage_stats]
    assert names == ["coarse:64", "coarse:128(active)", "finest:256(active)"], names
    assert act.active_rounds >= 1 and not act.active_fallback
    assert act.fw_error <= tol and act.penetration_error <= tol
    assert rel(act.pressure, full.pressure) <= 20 * tol
    assert rel(act.pressure, ora.pressure) <= 20 * tol
    assert abs(act.contact_area - full.contact_area) <= 1e-4
    assert abs(act.iterations - ora.iterations) <= max(3, ora.iterations // 4)
    # the fields come from the certifying apply: gap = u + g0 - approach
    gap = np.asarray(act.gap).ravel()
    u = np.asarray(act.displacement).ravel()
    assert np.max(np.abs(gap - (u + g - act.approach))) <= 1e-9 * np.max(np.abs(g))
    assert gap.min() >= -tol * max(g.max() - g.min(), pbar) * 1.01


def test_active_set_fallback_and_expansion():
    """A candidate set that misses contact: no halo and delta 0 leave out
    the points that the finer level brings into contact; one round then
    fails the global check and the full-grid fallback solve certifies."""
    import aspher_b200 as hc
    ns, pbar, tol = 256, 0.02, 1e-7
    g = hc.self_affine_gap(ns, hurst=0.8, rms=0.002, seed=5)
    kw = dict(coarsest=64, tol=tol, backend="fft", light_result=True)
    full = hc.solve_nested(ns, g, pbar, **kw)
    one = hc.solve_nested(ns, g, pbar, active_set=True, active_halo=0, active_delta=0.0,
                          active_max_rounds=1, **kw)
    assert one.status == "converged" and one.active_fallback and one.active_rounds == 1
    assert rel(one.pressure, full.pressure) <= 20 * tol
    many = hc.solve_nested(ns, g, pbar, active_set=True, active_halo=0, active_delta=0.0,
                           active_max_rounds=8, **kw)
    assert many.status == "converged"
    assert many.active_rounds > 1 or many.active_fallback
    assert rel(many.pressure, full.pressure) <= 20 * tol


@pytest.mark.parametrize("active", [False, True])
def test_nested_non_power_of_two_levels_match_oracle(active):
    """Ns = coarsest * 2^k with levels that are not powers of two (the
    reference accepts them, nested_solve.cpp:523-560): 25 -> 50 -> 100 run on
    embedded operators; the same result as the oracle's nested solve and as
    a single full-grid solve on the 100 x 100 grid."""
    import aspher_b200 as hc
    from oracle.api import solve_nested as osolve
    ns, pbar, tol = 100, 0.02, 1e-8
    g = _rough(ns, seed=7, rms=0.02, k_hi=16)
    r = hc.solve_nested(ns, g, pbar, coarsest=25, backend="fft", tol=tol,
                        precond_engine="stencil", active_set=active)
    o = osolve(ns, g, pbar, coarsest=25, backend="fft", tol=tol, precond_engine="stencil")
    assert r.status == "converged" and o.status == "converged", (r.status, r.status_reason)
    assert [st["name"].split(":")[1].split("(")[0] for st in r.stage_stats] == ["25", "50", "100"]
    assert rel(r.pressure, o.pressure) <= 10 * tol
    assert abs(r.contact_area - o.contact_area) <= 1e-4
    full = hc.ContactSolver(ns, backend="fft").solve(g, pbar, tol, precond="fourier")
    assert rel(r.pressure, full.pressure) <= 10 * tol
    with pytest.raises(ValueError, match="even levels"):
        hc.solve_nested(ns, g, pbar, coarsest=25, backend="periodic", tol=tol)
    # even levels: the periodic backend's default fft engine runs embedded
    rp = hc.solve_nested(ns, g, pbar, coarsest=50, backend="periodic", tol=tol)
    op_ = osolve(ns, g, pbar, coarsest=50, backend="periodic", tol=tol)
    assert rp.status == "converged" and op_.status == "converged"
    assert rel(rp.pressure, op_.pressure) <= 10 * tol
