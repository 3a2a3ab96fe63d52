"""Grids that are not powers of two (B200).

The reference's fft and periodic backends take any grid_size (its FFT
engine is pocketfft, src/fft_engine.hpp:147-290).  Here such an operator
runs embedded: its Nl x Nl cells are the top-left block of the free-space
pipeline of the next power of two, whose kernel table holds the Love table
at the caller's cell size (fft) or the real-space kernel of the periodic
symbol on the Nl torus (periodic).  Gates:

* operator: equal to the reference's own operator (oracle/_ref, else the
  numpy oracle, itself pinned to the reference at these sizes in
  test_ref_oracle.py) -- fft FP64 1e-13; periodic FP64 1e-12 (the kernel
  table is a sum of Nl^2 cosine terms, each entry correct to a few
  roundings of its largest term); FP32 2e-6;
* solves: status, pressure rel-L2 <= 10 tol, contact area within 1e-4 and
  the load exact against the reference's solve on the same grid, for both
  backends, unpreconditioned and with the stencil preconditioner (wrap at
  the caller's side), FP64, FP32 and float_then_double;
* batched and heterogeneous-batch solves reach the same pressures;
* the Love table API returns the caller's Nl x Nl table;
* what needs a power-of-two grid says so.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import ref  # noqa: E402
from oracle.api import ContactSolver as OSolver  # noqa: E402

pytestmark = pytest.mark.gpu


def _oracle(Ns, backend, L=1.0, E=1.0):
    if ref.available():
        return ref.ContactSolver(Ns, backend=backend, domain_size=L, E_star=E)
    return OSolver(Ns, backend=backend, domain_size=L, E_star=E)


def _rel(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _gap(Ns, seed=42, rms=0.002):
    from aspher_b200 import self_affine_gap
    return self_affine_gap(Ns, hurst=0.8, rms=rms, seed=seed)


@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("Ns", [2, 5, 12, 37, 100, 255, 1000])
def test_embedded_operator_matches_reference(backend, Ns):
    from aspher_b200 import ContactSolver, Operator
    L, E = 1.1, 1.3
    op = Operator(backend, Ns, L, E)
    assert op.info().grid_size == Ns and op.info().n == Ns * Ns
    x = np.random.default_rng(Ns + 1).standard_normal(Ns * Ns)
    want = _oracle(Ns, backend, L, E).matvec(x)
    got = np.asarray(ContactSolver(Ns, L, E, backend=backend).matvec(x)).ravel()
    assert got.shape == (Ns * Ns,)
    assert _rel(got, want) <= (1e-13 if backend == "fft" else 1e-12)
    x64 = torch.as_tensor(x, device="cuda")
    y64 = torch.empty_like(x64)
    op.matvec_(x64, y64)
    assert _rel(y64.cpu().numpy(), want) <= (1e-13 if backend == "fft" else 1e-12)
    x32 = torch.as_tensor(x, dtype=torch.float32, device="cuda")
    y32 = torch.empty_like(x32)
    op.matvec_(x32, y32)
    assert _rel(y32.double().cpu().numpy(), want) <= 2e-6


def test_embedded_love_table():
    from aspher_b200 import Operator
    Ns = 37
    got = Operator("fft", Ns, 2.0, 1.5).love_table()
    want = _oracle(Ns, "fft", 2.0, 1.5).love_table()
    assert got.shape == (Ns, Ns)
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-12


@pytest.mark.parametrize("precond", ["none", "fourier"])
@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("Ns", [100, 75])
def test_embedded_solve_matches_reference(Ns, backend, precond):
    from aspher_b200 import ContactSolver
    pbar, tol = 0.005, 1e-8
    g0 = _gap(Ns)
    r = ContactSolver(Ns, backend=backend).solve(g0, pbar, tol, 5000, precond=precond)
    o = _oracle(Ns, backend).solve(g0, pbar, tol, 5000, precond=precond)
    assert o.status == "converged"
    assert r.status == "converged", (r.status, r.status_reason)
    assert _rel(r.pressure, o.pressure) <= 10 * tol
    assert abs(r.contact_area - o.contact_area) <= 1e-4
    assert abs(r.mean_pressure - pbar) <= 1e-12 * pbar
    assert r.fw_error <= tol and r.penetration_error <= tol
    assert np.asarray(r.pressure).shape == (Ns, Ns)
    # the reference's own iteration count, up to the reduction-order slack
    # its tests allow (test_fft.cpp:89-95), a little wider with the stencil
    assert abs(r.iterations - o.iterations) <= (2 if precond == "none" else 6)
    u = np.asarray(r.displacement).ravel()
    assert _rel(u, _oracle(Ns, backend).matvec(np.asarray(r.pressure).ravel())) <= 1e-12


@pytest.mark.parametrize("precision", ["float", "float_then_double"])
def test_embedded_mixed_precision(precision):
    from aspher_b200 import ContactSolver
    Ns, pbar = 300, 0.005
    g0 = _gap(Ns)
    s = ContactSolver(Ns, backend="fft")
    rd = s.solve(g0, pbar, 1e-10, precond="fourier")
    tol = 1e-6 if precision == "float" else 1e-8
    r = s.solve(g0, pbar, tol, precond="fourier", precision=precision)
    assert rd.status == "converged" and r.status == "converged", (r.status, r.status_reason)
    assert _rel(r.pressure, rd.pressure) <= (1e-5 if precision == "float" else 1e-7)
    assert abs(r.contact_area - rd.contact_area) <= 1e-4


def test_embedded_batch_and_many():
    from aspher_b200 import Operator, solve_device, solve_device_batch
    from aspher_b200.batch import solve_many
    Ns, tol = 90, 1e-8
    op = Operator("fft", Ns)
    gs = [torch.as_tensor(_gap(Ns, seed=s), device="cuda") for s in (1, 2, 3)]
    loads = [0.002, 0.005, 0.01]
    single = [solve_device(op, g, p, tol=tol, precond="fourier") for g, p in zip(gs, loads)]
    batch = solve_device_batch(op, gs, loads, tol=tol, precond="fourier")
    for a, b in zip(single, batch):
        assert a.status == b.status == "converged"
        assert _rel(b.pressure_device.cpu().numpy(), a.pressure_device.cpu().numpy()) <= 1e-12
    probs = [dict(backend="fft", grid_size=Ns, p_nominal=loads[0]),
             dict(backend="periodic", grid_size=50, p_nominal=0.004),
             dict(backend="fft", grid_size=64, p_nominal=0.003)]
    gaps = [gs[0], _gap(50, seed=5), _gap(64, seed=6)]
    out = solve_many(probs, gaps, tol=tol, precision="double", precond="fourier")
    for pr, g, res in zip(probs, gaps, out):
        g = g.cpu().numpy() if torch.is_tensor(g) else g
        o = _oracle(pr["grid_size"], pr["backend"]).solve(g, pr["p_nominal"], tol,
                                                           precond="fourier")
        assert res.status == "converged"
        assert _rel(res.pressure_device.cpu().numpy(), o.pressure) <= 10 * tol


def test_embedded_rejects_what_needs_a_power_of_two():
    from aspher_b200 import ContactSolver, Operator
    s = ContactSolver(61, backend="fft")
    with pytest.raises(ValueError, match="even grid_size"):
        s.solve(_gap(61), 0.005, 1e-8, precond="fourier-fft")
    with pytest.raises(ValueError, match="power-of-two"):
        Operator("fft", 60, flags=1)
    with pytest.raises(ValueError):
        Operator("fft", 1)
    with pytest.raises(ValueError):
        Operator("periodic", 16385)


def test_embedded_warm_start_and_history():
    """p_init on an embedded grid: the caller's Nl^2 warm start (the
    converged pressure) is embedded with zero outside the block; the solve
    restarts at the optimum (the reference's test_certification.cpp:76-148
    warm start) and keeps its certificate; the error history has one entry
    per iteration."""
    from aspher_b200 import ContactSolver
    Ns, pbar, tol = 60, 0.005, 1e-8
    g0 = _gap(Ns)
    s = ContactSolver(Ns, backend="fft")
    r = s.solve(g0, pbar, tol, precond="fourier")
    assert r.status == "converged"
    w = s.solve(g0, pbar, tol, precond="fourier", p_init=np.asarray(r.pressure))
    assert w.status == "converged"
    assert w.iterations <= 2
    assert _rel(w.pressure, r.pressure) <= 10 * tol
    from aspher_b200 import Operator, solve_device
    op = Operator("periodic", 45)
    g = torch.as_tensor(_gap(45), device="cuda")
    h = solve_device(op, g, pbar, tol=tol, record_history=True, precond="fourier")
    assert h.status == "converged" and len(h.error_history) == h.iterations


@pytest.mark.parametrize("Ns,radius", [(50, 2), (37, 3), (200, 2)])
def test_embedded_stencil_preconditioner_matches_reference(Ns, radius):
    """The standalone stencil apply on an embedded grid wraps at the
    caller's side (stencil_precond.cpp:63-109 on the Nl torus) with the taps
    of min(Nl, 512); against the reference's own apply (oracle/_ref) where it
    is built, else the numpy restatement; FP64 1e-13, FP32 2e-6."""
    from aspher_b200 import Operator
    from oracle.precond import StencilPreconditioner
    rng = np.random.default_rng(5 + Ns)
    g = rng.standard_normal(Ns * Ns)
    c = (rng.random(Ns * Ns) < 0.35).astype(np.uint8)
    op = Operator("fft", Ns)
    if ref.available():
        want = ref.ContactSolver(Ns, backend="fft").precond_apply(g, c, "fourier", radius)
    else:
        want = StencilPreconditioner(Ns, radius).apply(g, c.astype(bool), np.float64)
    for dt, tol in ((torch.float64, 1e-13), (torch.float32, 2e-6)):
        gd = torch.as_tensor(g, dtype=dt, device="cuda")
        cd = torch.as_tensor(c, device="cuda")
        z = torch.empty_like(gd)
        op.precond_("stencil", gd, cd, z, radius=radius)
        got = z.cpu().numpy().astype(np.float64)
        assert np.all(got[c == 0] == 0.0)
        assert _rel(got, want) < tol


@pytest.mark.parametrize("Ns", [50, 100])
def test_embedded_fourier_preconditioner_matches_reference(Ns):
    """The full-grid |k| preconditioner on an even grid that is not a power
    of two: the circulant of the reference's float symbol |k| / Ns^2 on the
    Ns torus (fourier_precond.cpp:12-116) as a padded convolution with its
    real-space kernel.  Against the reference's own apply (oracle/_ref) or
    the numpy restatement: FP64 1e-12 (the kernel table is a cosine sum
    over Ns^2 terms), FP32 2e-6."""
    from aspher_b200 import Operator
    from oracle.precond import FourierPreconditioner
    rng = np.random.default_rng(17 + Ns)
    g = rng.standard_normal(Ns * Ns)
    c = (rng.random(Ns * Ns) < 0.35).astype(np.uint8)
    op = Operator("fft", Ns)
    if ref.available():
        want = ref.ContactSolver(Ns, backend="fft").precond_apply(g, c, "fourier-fft")
    else:
        want = FourierPreconditioner(Ns).apply(g, c.astype(bool), np.float64)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 2e-6)):
        gd = torch.as_tensor(g, dtype=dt, device="cuda")
        cd = torch.as_tensor(c, device="cuda")
        z = torch.empty_like(gd)
        op.precond_("fft", gd, cd, z)
        got = z.cpu().numpy().astype(np.float64)
        assert np.all(got[c == 0] == 0.0)
        assert _rel(got, want) < tol


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_embedded_solve_with_fourier_preconditioner(backend):
    from aspher_b200 import ContactSolver
    Ns, pbar, tol = 100, 0.005, 1e-8
    g0 = _gap(Ns)
    r = ContactSolver(Ns, backend=backend).solve(g0, pbar, tol, 5000, precond="fourier-fft")
    o = _oracle(Ns, backend).solve(g0, pbar, tol, 5000, precond="fourier-fft")
    assert o.status == "converged" and r.status == "converged", (r.status, r.status_reason)
    assert _rel(r.pressure, o.pressure) <= 10 * tol
    assert abs(r.contact_area - o.contact_area) <= 1e-4
    assert abs(r.iterations - o.iterations) <= 6
