"""Parity of the CUDA Polonsky-Keer solve with the oracle (B200).

Acceptance (the bar the north star states): status 'converged', pressure
rel-L2 vs the oracle's FP64 solve <= 10 * tol (1e-5 absolute floor for the
FP32 path, whose certificate floor is ~2e-7), |delta contact_area| <= 1e-4.
Iteration counts are compared loosely: the reference itself allows +-1 from
reduction order (tests/test_fft.cpp:89-95).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle.api import ContactSolver as OSolver  # noqa: E402
from oracle.operators import PeriodicFFTOperator as OPer  # noqa: E402
from oracle.solver import SolveOptions, solve_contact_impl  # noqa: E402

pytestmark = pytest.mark.gpu


def _solver(Ns, backend, L=1.0, E=1.0):
    from aspher_b200 import ContactSolver
    return ContactSolver(Ns, domain_size=L, E_star=E, backend=backend)


def _rough(Ns, seed=42, rms=0.002):
    from aspher_b200 import self_affine_gap
    return self_affine_gap(Ns, hurst=0.8, rms=rms, seed=seed)


def _hertz(Ns, R=0.5):
    h = 1.0 / Ns
    x = (np.arange(Ns) + 0.5) * h - 0.5
    return ((x[None, :] ** 2 + x[:, None] ** 2) / (2 * R)).ravel()


def rel(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_hertz_fft_matches_oracle():
    Ns, pbar = 64, 0.05
    g0 = _hertz(Ns)
    r = _solver(Ns, "fft").solve(g0, pbar, 1e-8, 2000)
    o = OSolver(Ns, backend="fft").solve(g0, pbar, 1e-8, 2000)
    assert r.status == "converged" and o.status == "converged"
    assert abs(r.iterations - o.iterations) <= 1
    assert r.contact_area == o.contact_area
    assert rel(r.pressure, o.pressure) < 1e-6
    assert abs(r.mean_pressure - pbar) < 1e-12 * pbar


@pytest.mark.parametrize("precond", ["none", "fourier", "fourier-fft"])
@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_rough_solve_matches_oracle(backend, precond):
    Ns, pbar, tol = 128, 0.005, 1e-8
    g0 = _rough(Ns)
    r = _solver(Ns, backend).solve(g0, pbar, tol, 5000, precond=precond)
    o = OSolver(Ns, backend=backend).solve(g0, pbar, tol, 5000, precond=precond)
    assert r.status == "converged", (r.status, r.status_reason, r.iterations)
    assert o.status == "converged"
    assert r.fw_error <= tol and r.penetration_error <= tol
    assert rel(r.pressure, o.pressure) <= 10 * tol
    assert abs(r.contact_area - o.contact_area) <= 1e-4
    assert abs(r.iterations - o.iterations) <= max(3, o.iterations // 10)
    assert r.precond_count == (0 if precond == "none" else r.precond_count)
    assert r.pressure.min() >= 0.0


def test_westergaard_gpu():
    n, L, Es, D = 256, 2.0, 1.3, 0.01
    pstar = np.pi * Es * D / L
    s = _solver(n, "periodic", L, Es)
    cosx = np.tile(np.cos(2 * np.pi * np.arange(n) / n), (n, 1)).ravel()
    g0 = D * (1 - cosx)
    r = s.solve(g0, 1.5 * pstar, 1e-12)
    assert r.status == "converged"
    pex = 1.5 * pstar + pstar * cosx
    assert rel(r.pressure, pex) < 1e-9
    r = s.solve(g0, 0.3 * pstar, 1e-10)
    assert r.status == "converged"
    width = (r.pressure.ravel()[:n] > 0).sum() * L / n
    wex = 2 * (L / np.pi) * np.arcsin(np.sqrt(0.3))
    assert abs(width - wex) <= 2 * L / n


def test_status_taxonomy():
    """test_certification.cpp:215-323 (T03)."""
    Ns = 32
    g0 = _hertz(Ns)
    s = _solver(Ns, "fft")
    r = s.solve(g0, 0.02, 1e-8, max_iter=0)
    assert r.status == "max_iterations" and r.iterations == 0
    r = s.solve(g0, 0.02, 1e-8, max_iter=1)
    assert r.status in ("max_iterations", "converged") and r.iterations <= 1
    r = s.solve(g0, 0.02, 1e-25, max_iter=300)
    assert r.status in ("stagnated", "max_iterations", "converged")
    if r.status == "converged":
        assert r.fw_error <= 1e-15 and r.penetration_error <= 1e-15
    bad = g0.copy()
    bad[5] = np.nan
    with pytest.raises(ValueError):
        s.solve(bad, 0.02, 1e-8)
    with pytest.raises(ValueError):
        s.solve(g0, -1.0, 1e-8)
    with pytest.raises(ValueError):
        s.solve(g0, 0.02, 0.0)
    with pytest.raises(ValueError):
        s.solve(g0, 0.02, 1e-8, max_iter=-1)


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_binding_surface_for_fourier_backends(backend):
    """bindings.cpp:240-260: block_layout is (0, 6) and recompress a no-op for
    every backend but 'hmatrix'; hmatrix_info names the backend."""
    s = _solver(16, backend)
    bl = s.block_layout()
    assert bl.shape == (0, 6) and bl.dtype == np.float64
    x = np.random.default_rng(3).standard_normal(256)
    u0 = s.matvec(x)
    assert s.recompress(1e-4) is None
    assert np.array_equal(s.matvec(x), u0)
    info = s.hmatrix_info()
    assert info["backend"] == backend and info["n"] == 256


def test_singleton_warm_start_repaired():
    """test_certification_py.py:42-73 on the fft backend."""
    ns = 16
    x = (np.arange(ns) + 0.5) / ns - 0.5
    g0 = (x[:, None] ** 2 + x[None, :] ** 2).ravel()
    s = _solver(ns, "fft")
    warm = np.zeros(ns * ns)
    warm[0] = 0.01 * ns * ns
    cold = s.solve(g0, 0.01, tol=1e-10)
    got = s.solve(g0, 0.01, tol=1e-10, p_init=warm)
    assert got.status == "converged" and got.iterations > 0
    assert rel(got.pressure, cold.pressure) < 1e-6


def test_gap_datum_invariance():
    """A large additive gap offset must not change the pressure (T07)."""
    Ns = 64
    g0 = _rough(Ns)
    s = _solver(Ns, "fft")
    ref = s.solve(g0, 0.02, 1e-10, precond="fourier")
    for shift in (1e3, 1e6):
        r = s.solve(g0 + shift, 0.02, 1e-10, precond="fourier")
        assert r.status == "converged"
        assert rel(r.pressure, ref.pressure) < 1e-7
        assert abs(r.approach - ref.approach - shift) < 1e-6 * max(1.0, shift)


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_float_solve_matches_double(backend):
    Ns, pbar, tol = 256, 0.005, 1e-6
    g0 = _rough(Ns)
    s = _solver(Ns, backend)
    rd = s.solve(g0, pbar, 1e-10, precond="fourier")
    rf = s.solve(g0, pbar, tol, precond="fourier", precision="float")
    assert rf.status == "converged", (rf.status, rf.status_reason)
    assert rel(rf.pressure, rd.pressure) <= 1e-5
    assert abs(rf.contact_area - rd.contact_area) <= 1e-4
    rp = s.solve(g0, pbar, 1e-8, precond="fourier", precision="float_then_double")
    assert rp.status == "converged"
    assert rel(rp.pressure, rd.pressure) <= 1e-7


def test_history_and_counts():
    Ns = 64
    from aspher_b200 import Operator, solve_device
    op = Operator("fft", Ns)
    g0 = torch.as_tensor(_rough(Ns), device="cuda")
    r = solve_device(op, g0, 0.01, tol=1e-8, record_history=True, precond="fourier")
    assert r.status == "converged"
    assert len(r.error_history) == r.iterations
    assert r.matvec_count >= 2 * r.iterations
    assert r.precond_count >= 1


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_polish_reaches_fp64_certificates(backend):
    """The FP64 polish stage applies S defect-corrected (FP32 transforms of
    p - p0 and of the direction around one exact FP64 apply of p0); it still
    certifies FP64 tolerances, and the result matches a tight FP64 solve."""
    from aspher_b200 import Operator, solve_device, solve_device_mixed
    Ns, pbar = 256, 0.005
    op = Operator(backend, Ns)
    g0 = torch.as_tensor(_rough(Ns), device="cuda")
    ref = solve_device(op, g0, pbar, tol=1e-12, precond="fourier", dtype=torch.float64,
                       max_iter=20000)
    assert ref.status == "converged"
    r, rf = solve_device_mixed(op, g0, pbar, tol=1e-10, float_tol=1e-5, precond="fourier")
    assert rf.status == "converged" and rf.fw_error <= 1e-5
    assert r.status == "converged", (r.status, r.status_reason)
    assert r.fw_error <= 1e-10 and r.penetration_error <= 1e-10
    assert rel(r.pressure, ref.pressure) <= 1e-8


@pytest.mark.parametrize("precision", ["float", "float_then_double"])
def test_mixed_result_states_its_accuracy_vs_fp64(precision):
    """solve(..., reference_fp64=True) runs the plain FP64 solve beside the
    float / float_then_double one and reports the pressure rel-L2 and the
    contact-area error against it; without the flag the fields are None."""
    Ns, pbar, tol = 256, 0.005, 1e-6
    g0 = _rough(Ns)
    s = _solver(Ns, "fft")
    r = s.solve(g0, pbar, tol, precond="fourier", precision=precision, reference_fp64=True)
    rd = s.solve(g0, pbar, tol, precond="fourier")
    assert r.status == "converged" and r.fp64_status == rd.status == "converged"
    assert r.pressure_rel_l2_vs_fp64 == pytest.approx(rel(r.pressure, rd.pressure), rel=1e-6,
                                                      abs=1e-12)
    assert r.contact_area_error_vs_fp64 == pytest.approx(abs(r.contact_area - rd.contact_area),
                                                         abs=1e-12)
    assert r.pressure_rel_l2_vs_fp64 <= 1e-4 and r.contact_area_error_vs_fp64 <= 1e-4
    plain = s.solve(g0, pbar, tol, precond="fourier", precision=precision)
    assert plain.pressure_rel_l2_vs_fp64 is None and plain.contact_area_error_vs_fp64 is None


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_eager_loop_matches_graph_loop(dtype):
    """loop_mode="eager" launches the loop body's kernels one by one with the
    while condition read on the host: the same kernels in the same order, so
    the same iterates bit for bit (FP64 and FP32, stencil preconditioner,
    the mixed float_then_double path included)."""
    from aspher_b200 import Operator, solve_device, solve_device_mixed
    Ns, pbar = 128, 0.005
    op = Operator("fft", Ns)
    g0 = torch.as_tensor(_rough(Ns), device="cuda")
    dt = torch.float64 if dtype == "f64" else torch.float32
    tol = 1e-8 if dtype == "f64" else 1e-6
    a = solve_device(op, g0, pbar, tol=tol, precond="fourier", dtype=dt)
    b = solve_device(op, g0, pbar, tol=tol, precond="fourier", dtype=dt, loop_mode="eager")
    assert a.status == b.status == "converged"
    assert a.iterations == b.iterations and a.matvec_count == b.matvec_count
    assert torch.equal(a.pressure_device, b.pressure_device)
    if dtype == "f64":
        ma, _ = solve_device_mixed(op, g0, pbar, tol=1e-8, precond="fourier")
        mb, _ = solve_device_mixed(op, g0, pbar, tol=1e-8, precond="fourier", loop_mode="eager")
        assert ma.iterations == mb.iterations
        assert torch.equal(ma.pressure_device, mb.pressure_device)
    with pytest.raises(ValueError):
        solve_device(op, g0, pbar, loop_mode="stream")
