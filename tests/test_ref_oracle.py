"""The numpy oracle against the reference's own C++ (CPU, no GPU).

``oracle/_ref/libaspher_ref.so`` is the reference's unmodified hot-path
sources (src/contact_solver.cpp, src/fft_operator.cpp,
src/periodic_fft_operator.cpp, src/boussinesq_kernel.cpp,
src/stencil_precond.cpp, src/fourier_precond.cpp) compiled against the
project's Eigen-API shim (``make -C oracle``).  These tests pin the numpy
restatement in ``oracle/`` -- the checker the GPU parity tests use -- to the
reference itself: operators, preconditioners, the projector and whole PK
solves agree to rounding, with equal iteration counts and statuses.  They
are skipped where the library has not been built (it needs the reference
tree).
"""

import numpy as np
import pytest

from oracle import ref
from oracle.api import ContactSolver as OracleSolver
from oracle.precond import FourierPreconditioner, StencilPreconditioner
from oracle.solver import project_load_simplex

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _gap(Ns, seed=42, rms=0.002):
    from aspher_b200.surfaces import self_affine_gap
    return self_affine_gap(Ns, hurst=0.8, rms=rms, seed=seed)


def _rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


@needs_ref
@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("Ns", [16, 32, 64])
def test_matvec_matches_reference(backend, Ns):
    """FFTOperator / PeriodicFFTOperator matvec_into and matvec_single_into."""
    a, b = ref.ContactSolver(Ns, backend=backend, domain_size=1.3, E_star=0.7), OracleSolver(
        Ns, backend=backend, domain_size=1.3, E_star=0.7)
    x = np.random.default_rng(Ns).standard_normal(Ns * Ns)
    assert _rel(a.matvec(x), b.matvec(x)) <= 1e-14
    y32 = a.matvec(x.astype(np.float32), dtype=np.float32)
    assert _rel(y32.astype(np.float64), b.matvec(x)) <= 2e-6


@needs_ref
def test_love_table_matches_reference():
    """BoussinesqKernel table (src/boussinesq_kernel.cpp:97-106)."""
    from oracle.love import boussinesq_table
    Ns = 48
    t = ref.ContactSolver(Ns, backend="fft", domain_size=2.0, E_star=1.5).love_table()
    o = boussinesq_table(Ns, 2.0, 1.5)
    # the reference's own gate for its kernel (test_kernel_stability.cpp:53-83):
    # the far-field asinh differences cancel to a few 1e-14
    assert np.max(np.abs(t - o) / np.abs(o)) <= 1e-12


@needs_ref
@pytest.mark.parametrize("precond", ["fourier", "fourier-fft"])
def test_preconditioners_match_reference(precond):
    """StencilPreconditioner::apply_into / FourierPreconditioner::apply_into."""
    Ns = 64
    rng = np.random.default_rng(3)
    g = rng.standard_normal(Ns * Ns)
    c = (rng.random(Ns * Ns) < 0.3).astype(np.uint8)
    a = ref.ContactSolver(Ns, backend="periodic")
    z = a.precond_apply(g, c, precond=precond)
    if precond == "fourier":
        zo = StencilPreconditioner(Ns, 2).apply(g, c, np.float64)
    else:
        zo = FourierPreconditioner(Ns).apply(g, c, np.float64)
    assert _rel(z, zo) <= 1e-13


@needs_ref
def test_simplex_projector_matches_reference():
    """project_load_simplex (src/contact_solver.cpp:31-60)."""
    y = np.random.default_rng(5).standard_normal(1000)
    pr, th = ref.project_load_simplex(y, 7.5)
    po = y.copy()
    tho = project_load_simplex(po, 7.5)
    assert abs(th - tho) <= 1e-13 * max(1.0, abs(th))
    assert np.max(np.abs(pr - po)) <= 1e-13
    assert abs(pr.sum() - 7.5) <= 1e-12


@needs_ref
@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("precond", ["none", "fourier", "fourier-fft"])
def test_solve_matches_reference(backend, precond):
    """solve_contact (src/contact_solver.cpp:150-587, 1071-1082): same
    status, iterations and certificates; pressure to rounding."""
    Ns = 64
    g = _gap(Ns)
    a = ref.ContactSolver(Ns, backend=backend).solve(g, 0.005, tol=1e-8, precond=precond)
    b = OracleSolver(Ns, backend=backend).solve(g, 0.005, tol=1e-8, precond=precond)
    assert a.status == b.status == "converged"
    assert a.iterations == b.iterations
    assert a.identification_steps == b.identification_steps
    assert _rel(a.pressure, b.pressure) <= 1e-12
    assert a.contact_area == b.contact_area
    for k in ("fw_error", "penetration_error", "approach", "objective"):
        assert abs(getattr(a, k) - getattr(b, k)) <= 1e-9 * max(1.0, abs(getattr(b, k))), k


@needs_ref
def test_config1_reference_solve_matches_oracle():
    """The plain-method configuration (fft, Ns=256, FP64, seed 42, p_nominal
    0.005, tol 1e-8, precond "fourier"): the numpy oracle reproduces the
    reference's own solve."""
    Ns = 256
    g = _gap(Ns)
    a = ref.ContactSolver(Ns, backend="fft").solve(g, 0.005, tol=1e-8, precond="fourier")
    b = OracleSolver(Ns, backend="fft").solve(g, 0.005, tol=1e-8, precond="fourier")
    assert a.status == b.status == "converged"
    assert a.iterations == b.iterations
    assert _rel(a.pressure, b.pressure) <= 1e-12


@needs_ref
def test_float_solve_matches_reference():
    """solve_contact_impl<float> (the float stage of the nested driver) on
    the reference vs the oracle's float path: both certify, and their
    pressures agree far inside the float floor."""
    from oracle.solver import SolveOptions, solve_contact_impl
    from oracle.operators import FFTOperator
    Ns = 64
    g = _gap(Ns)
    a = ref.ContactSolver(Ns, backend="fft").solve(g, 0.005, tol=1e-6, precond="fourier",
                                                    dtype=np.float32)
    op = FFTOperator(Ns)
    sp = StencilPreconditioner(Ns, 2)
    b = solve_contact_impl(lambda x: op.matvec(x, np.float32), g.reshape(-1), 0.005,
                           SolveOptions(tol=1e-6), lambda gg, c: sp.apply(gg, c, np.float32),
                           None, dtype=np.float32)
    assert a.status == b.status == "converged"
    assert abs(a.iterations - b.iterations) <= 3
    assert _rel(a.pressure, b.pressure) <= 2e-5


STALL_CASES = [
    # (backend, Ns, p_nominal): with stall_limit 1 and no preconditioner the
    # merit stalls early, so the stall forces identification steps
    # (src/contact_solver.cpp:383-407); the first ends `stagnated` / "stall"
    # after three of them, the second converges after two
    ("fft", 64, 0.02),
    ("periodic", 32, 0.02),
]


@needs_ref
@pytest.mark.parametrize("backend,Ns,pbar", STALL_CASES)
def test_stall_forced_identification_matches_reference(backend, Ns, pbar):
    """Stall-forced identification steps: the oracle takes the reference's
    branch with the same counts, status, reason and pressure."""
    from oracle.solver import SolveOptions, solve_contact_impl
    from oracle.operators import FFTOperator, PeriodicFFTOperator
    g = _gap(Ns)
    a = ref.ContactSolver(Ns, backend=backend).solve(g, pbar, tol=1e-10, max_iter=3000,
                                                      stall_limit=1)
    op = FFTOperator(Ns) if backend == "fft" else PeriodicFFTOperator(Ns)
    b = solve_contact_impl(lambda x: op.matvec(x, np.float64), g.reshape(-1), pbar,
                           SolveOptions(tol=1e-10, max_iter=3000, stall_limit=1), None, None,
                           dtype=np.float64)
    assert a.identification_steps >= 2
    assert a.status == b.status
    assert a.status_reason == b.status_reason
    assert a.identification_steps == b.identification_steps
    assert a.iterations == b.iterations
    assert a.returned_best == b.returned_best
    assert _rel(a.pressure, b.pressure) <= 1e-12


def test_oracle_iterations_at_ns2048_equal_reference():
    """At the benchmark size the numpy oracle's FP64 solves take exactly the
    reference's iterations and reach its contact areas (the oracle's counts
    in bench_iterations.json, the reference's in ref_ns2048.json; both made
    by the generator scripts beside them)."""
    import json
    import os
    golden = os.path.join(os.path.dirname(__file__), "golden")
    with open(os.path.join(golden, "bench_iterations.json")) as f:
        ours = json.load(f)["problems"]
    with open(os.path.join(golden, "ref_ns2048.json")) as f:
        theirs = json.load(f)["problems"]
    assert set(ours) == set(theirs)
    for k in ours:
        assert ours[k]["iterations"] == theirs[k]["tol6"]["iterations"], k
        assert ours[k]["status"] == theirs[k]["tol6"]["status"] == "converged", k
        assert abs(ours[k]["contact_area"] - theirs[k]["tol6"]["contact_area"]) <= 1e-6, k


@needs_ref
@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("Ns", [5, 12, 37, 100])
def test_matvec_matches_reference_any_size(backend, Ns):
    """Grids that are not powers of two (the reference's pocketfft engine
    takes any n, src/fft_engine.hpp:147-290): the numpy oracle equals the
    reference's own operators there too."""
    a = ref.ContactSolver(Ns, backend=backend, domain_size=1.1, E_star=1.3)
    b = OracleSolver(Ns, backend=backend, domain_size=1.1, E_star=1.3)
    x = np.random.default_rng(Ns + 1).standard_normal(Ns * Ns)
    assert _rel(a.matvec(x), b.matvec(x)) <= 1e-14
