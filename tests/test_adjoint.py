"""Derivatives of the contact solve.

The reference has no derivative of its solve; the oracle is central finite
differences of the FP64 solve.  The CPU tests pin the dense adjoint of
``oracle/adjoint.py`` to finite differences of the oracle solve; the GPU
tests check ``aspher_adjoint`` (FP64 and FP32 CG) against the dense adjoint
on the same converged pressure, and the ``contact_pressure`` autograd
Function against finite differences of the CUDA FP64 solve.

Loss (the differentiation workload): a smoothed contact area plus a
pressure energy, L(p) = sum sigmoid(p / 1e-4) / N^2 + 0.5 mean(p^2).
Finite differences: directions d with unit RMS, step h = 1e-6 * rms(gap).
"""

import numpy as np
import pytest

from oracle.adjoint import adjoint_dense, operator_matrix
from oracle.api import ContactSolver as OSolver
from aspher_b200.surfaces import self_affine_gap

SIG = 1e-4


def loss_np(p):
    p = np.asarray(p, np.float64).ravel()
    N = p.size
    return float(np.sum(1.0 / (1.0 + np.exp(-p / SIG))) / N ** 2 + 0.5 * np.mean(p ** 2))


def dloss_np(p):
    p = np.asarray(p, np.float64).ravel()
    N = p.size
    s = 1.0 / (1.0 + np.exp(-p / SIG))
    return s * (1.0 - s) / (SIG * N ** 2) + p / N


def _gap(Ns, seed=7):
    return self_affine_gap(Ns, hurst=0.8, rms=0.002, k_lo=1.0, k_hi=Ns / 2, seed=seed)


@pytest.mark.parametrize("backend", ["periodic", "fft"])
def test_oracle_adjoint_matches_finite_differences(backend):
    Ns, pbar = 12, 0.004
    s = OSolver(Ns, backend=backend)
    g0 = _gap(Ns)
    tol = 1e-14
    r = s.solve(g0, pbar, tol=tol, max_iter=20000, precond="none")
    assert r.status == "converged"
    p = np.asarray(r.pressure).ravel()
    assert 2 < np.count_nonzero(p) < p.size
    S = operator_matrix(s.matvec, Ns * Ns)
    grad, dLdP = adjoint_dense(S, p, dloss_np(p))
    rms = float(np.sqrt(np.mean(g0 ** 2)))
    h = 1e-6 * rms
    rng = np.random.default_rng(100)

    def L_of(g, pb=pbar):
        rr = s.solve(g, pb, tol=tol, max_iter=20000, precond="none")
        assert rr.status == "converged"
        return loss_np(rr.pressure)

    for _ in range(4):
        d = rng.standard_normal(g0.size)
        d /= np.sqrt(np.mean(d ** 2))
        fd = (L_of(g0 + h * d) - L_of(g0 - h * d)) / (2 * h)
        ad = float(grad @ d)
        assert abs(fd - ad) <= 1e-4 * abs(ad) + 1e-12, (fd, ad)
    hp = 1e-6 * pbar
    fdp = (L_of(g0, pbar + hp) - L_of(g0, pbar - hp)) / (2 * hp)
    adp = dLdP * Ns * Ns
    assert abs(fdp - adp) <= 1e-4 * abs(adp), (fdp, adp)


# ---- GPU --------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("backend", ["periodic", "fft"])
@pytest.mark.parametrize("dt,bound", [("f64", 1e-8), ("f32", 1e-4)])
@pytest.mark.parametrize("precond", ["fourier", "none"])
@pytest.mark.parametrize("Ns", [32, 30])
def test_gpu_adjoint_matches_dense(backend, dt, bound, precond, Ns):
    """Ns = 30 runs embedded (the caller's block of a 32 x 32 grid)."""
    torch = pytest.importorskip("torch")
    from aspher_b200 import ContactSolver, adjoint
    pbar = 0.005
    s = ContactSolver(Ns, backend=backend)
    g0 = _gap(Ns, seed=3)
    r = s.solve(g0, pbar, tol=1e-12, max_iter=20000, precond="fourier")
    assert r.status == "converged"
    p = torch.as_tensor(r.pressure.ravel(), device="cuda")
    w = torch.as_tensor(dloss_np(r.pressure), device="cuda")
    grad, dpb, info = adjoint(s.op, p, w, tol=1e-12 if dt == "f64" else 1e-6,
                              precond=precond,
                              dtype=torch.float64 if dt == "f64" else torch.float32)
    assert info["status"] == "converged", info
    o = OSolver(Ns, backend=backend)
    S = operator_matrix(o.matvec, Ns * Ns)
    gref, dPref = adjoint_dense(S, r.pressure, dloss_np(r.pressure))
    ga = grad.cpu().numpy()
    assert np.linalg.norm(ga - gref) <= bound * np.linalg.norm(gref)
    assert abs(dpb - dPref * Ns * Ns) <= bound * abs(dPref * Ns * Ns) + 1e-14


@pytest.mark.gpu
def test_contact_pressure_autograd_matches_finite_differences():
    torch = pytest.importorskip("torch")
    from aspher_b200 import ContactSolver, contact_pressure, solve_device
    Ns, pbar = 64, 0.005
    s = ContactSolver(Ns, backend="periodic")
    g0 = torch.as_tensor(_gap(Ns, seed=11), device="cuda")
    gap = g0.clone().requires_grad_(True)
    pn = torch.tensor(pbar, dtype=torch.float64, requires_grad=True)
    p = contact_pressure(s, gap, pn, tol=1e-12, max_iter=20000)
    N = Ns * Ns
    L = torch.sum(torch.sigmoid(p / SIG)) / N ** 2 + 0.5 * torch.mean(p ** 2)
    L.backward()
    gg = gap.grad.detach().cpu().numpy()
    gp = float(pn.grad)

    def L_of(g, pb=pbar):
        r = solve_device(s.op, g, pb, tol=1e-12, max_iter=20000, precond="fourier",
                         dtype=torch.float64, light=True)
        assert r.status == "converged"
        return loss_np(r.pressure)

    rms = float(torch.sqrt(torch.mean(g0 ** 2)))
    h = 1e-6 * rms
    rng = np.random.default_rng(100)
    for _ in range(4):
        d = rng.standard_normal(N)
        d /= np.sqrt(np.mean(d ** 2))
        dd = torch.as_tensor(d, device="cuda")
        fd = (L_of(g0 + h * dd) - L_of(g0 - h * dd)) / (2 * h)
        ad = float(gg.ravel() @ d)
        assert abs(fd - ad) <= 1e-4 * abs(ad), (fd, ad)
    hp = 1e-6 * pbar
    fdp = (L_of(g0, pbar + hp) - L_of(g0, pbar - hp)) / (2 * hp)
    assert abs(fdp - gp) <= 1e-4 * abs(gp), (fdp, gp)
