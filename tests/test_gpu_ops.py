"""Parity of the CUDA operators and preconditioners with the oracle (B200).

Tolerances are the reference's own gates where it has one:
FFT matvec vs dense (tests/test_fft.cpp:20-39): FP64 < 1e-12, FP32 < 1e-5;
periodic Fourier modes (tests/test_periodic.cpp:16-36): < 2e-13;
repeat calls bitwise equal (test_fft.cpp:46-59, test_periodic.cpp:38-51).
Against the oracle (same algorithm, different reduction/FFT order) FP64
agrees to 1e-13 relative and FP32 to 2e-6 relative.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle.love import assemble_dense, boussinesq_table  # noqa: E402
from oracle.operators import FFTOperator as OFFT, PeriodicFFTOperator as OPer  # noqa: E402
from oracle.precond import FourierPreconditioner, StencilPreconditioner  # noqa: E402

pytestmark = pytest.mark.gpu


def _op(backend, Ns, L=1.0, E=1.0):
    from aspher_b200 import Operator
    return Operator(backend, Ns, L, E)


def _mv(op, x, dtype):
    xt = torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device="cuda")
    y = torch.empty_like(xt)
    op.matvec_(xt, y)
    torch.cuda.synchronize()
    return y.cpu().numpy().astype(np.float64)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_love_table_matches_oracle():
    Ns, L, E = 64, 1.0, 1.7
    T = _op("fft", Ns, L, E).love_table()
    ref = boussinesq_table(Ns, L, E)
    assert np.max(np.abs(T - ref) / np.abs(ref)) < 1e-13
    h = L / Ns
    exact = 4.0 * h * np.log(1.0 + np.sqrt(2.0)) / (np.pi * E)
    assert abs(T[0, 0] / exact - 1.0) < 1e-14  # test_kernel.cpp:21-24


@pytest.mark.parametrize("Ns", [16, 32, 64])
def test_fft_matvec_equals_dense(Ns):
    S = assemble_dense(Ns, 1.0, 1.0)
    op = _op("fft", Ns)
    x = np.random.default_rng(Ns).uniform(-1, 1, Ns * Ns)
    ref = S @ x
    assert rel(_mv(op, x, torch.float64), ref) < 1e-12
    assert rel(_mv(op, x.astype(np.float32), torch.float32), ref) < 1e-5
    assert op.info().max_im_ratio < 1e-10


@pytest.mark.parametrize("Ns", [128, 256, 512, 1024, 2048])
def test_fft_matvec_matches_oracle(Ns):
    op = _op("fft", Ns, 1.0, 1.0)
    ref_op = OFFT(Ns, 1.0, 1.0)
    x = np.random.default_rng(7).standard_normal(Ns * Ns)
    y64 = _mv(op, x, torch.float64)
    assert rel(y64, ref_op.matvec(x)) < 1e-13
    x32 = x.astype(np.float32)
    y32 = _mv(op, x32, torch.float32)
    assert rel(y32, ref_op.matvec(x32.astype(np.float64))) < 2e-6


def test_fft_repeat_calls_bitwise():
    op = _op("fft", 256)
    rng = np.random.default_rng(1)
    x, other = rng.standard_normal(256 * 256), rng.standard_normal(256 * 256)
    for dt in (torch.float64, torch.float32):
        y1 = _mv(op, x, dt)
        _mv(op, other, dt)
        assert np.array_equal(y1, _mv(op, x, dt))


def test_periodic_modes_exact():
    n, L, Es = 32, 3.0, 2.5
    op = _op("periodic", n, L, Es)
    ix = np.arange(n)
    for mx, my in ((1, 0), (0, 3), (2, 5)):
        q = 2 * np.pi * np.hypot(mx, my) / L
        p = np.cos(2 * np.pi * (mx * ix[None, :] + my * ix[:, None]) / n).ravel()
        assert rel(_mv(op, p, torch.float64), 2.0 / (Es * q) * p) < 2e-13
    ones = np.ones(n * n)
    assert np.linalg.norm(_mv(_op("periodic", n), ones, torch.float64)) < 1e-13


@pytest.mark.parametrize("Ns", [16, 64, 256, 1024, 2048])
def test_periodic_matches_oracle(Ns):
    op = _op("periodic", Ns, 1.7, 0.8)
    ref_op = OPer(Ns, 1.7, 0.8)
    x = np.random.default_rng(Ns).standard_normal(Ns * Ns)
    assert rel(_mv(op, x, torch.float64), ref_op.matvec(x)) < 1e-13
    x32 = x.astype(np.float32)
    assert rel(_mv(op, x32, torch.float32), ref_op.matvec(x32.astype(np.float64))) < 2e-6


@pytest.mark.parametrize("n", [7, 12, 16])
def test_periodic_matrix_properties_and_alias(n):
    """test_periodic.cpp:53-88 on its grids (7 and 12 run embedded, as the
    circulant of the Nl torus inside a power-of-two free-space pipeline):
    symmetric, PSD, circulant, null space = constants; x == y aliasing."""
    op = _op("periodic", n, 1.7, 0.8)
    N = n * n
    E = torch.eye(N, dtype=torch.float64, device="cuda")
    S = np.zeros((N, N))
    y = torch.empty(N, dtype=torch.float64, device="cuda")
    for j in range(N):
        op.matvec_(E[j].clone(), y)  # a fresh (aligned) buffer: rows of E sit at 8 N j bytes
        S[:, j] = y.cpu().numpy()
    assert np.linalg.norm(S - S.T) / np.linalg.norm(S) < 1e-14
    ev = np.linalg.eigvalsh(S)
    assert ev[0] > -1e-13 * ev[-1] and ev[1] > 1e-6 * ev[-1]
    sx, sy = 3 % n, 5 % n
    for iy in range(n):
        for ix in range(n):
            a = iy * n + ix
            b = ((iy - sy) % n) * n + (ix - sx) % n
            assert abs(S[a, sy * n + sx] - S[b, 0]) < 1e-14 * S[0, 0]
    x = torch.as_tensor(np.random.default_rng(0).standard_normal(N), device="cuda")
    ref = torch.empty_like(x)
    op.matvec_(x, ref)
    op.matvec_(x, x)  # aliased
    assert torch.linalg.norm(x - ref) <= 1e-15 * torch.linalg.norm(ref)
    xf = torch.as_tensor(np.random.default_rng(0).standard_normal(N), device="cuda")
    xf = xf.float()
    op.matvec_(xf, xf)  # aliased, float
    assert torch.linalg.norm(xf.double() - ref) < 2e-6 * torch.linalg.norm(ref)


def test_periodic_modes_exact_odd_grid():
    """test_periodic.cpp:16-36 on an odd grid (embedded): a cosine mode is an
    eigenvector with eigenvalue 2 / (E* |q|); constants map to 0."""
    n, L, Es = 27, 3.0, 2.5
    op = _op("periodic", n, L, Es)
    ix = np.arange(n)
    for mx, my in ((1, 0), (0, 3), (2, 5)):
        q = 2 * np.pi * np.hypot(mx, my) / L
        p = np.cos(2 * np.pi * (mx * ix[None, :] + my * ix[:, None]) / n).ravel()
        assert rel(_mv(op, p, torch.float64), 2.0 / (Es * q) * p) < 2e-13
    assert np.linalg.norm(_mv(op, np.ones(n * n), torch.float64)) < 1e-13


@pytest.mark.parametrize("kind,radius", [("stencil", 1), ("stencil", 2), ("stencil", 3),
                                          ("stencil", 4), ("fourier-fft", 2)])
@pytest.mark.parametrize("Ns", [64, 128, 512])
def test_preconditioners_match_oracle(kind, radius, Ns):
    # Ns = 64 runs the tiled stencil kernel, Ns >= 128 the register-window one
    rng = np.random.default_rng(11)
    g = rng.standard_normal(Ns * Ns)
    c = (rng.random(Ns * Ns) < 0.35).astype(np.uint8)
    op = _op("periodic", Ns)
    P = StencilPreconditioner(Ns, radius) if kind == "stencil" else FourierPreconditioner(Ns)
    for dt, tol in ((torch.float64, 1e-13), (torch.float32, 2e-6)):
        npdt = np.float64 if dt == torch.float64 else np.float32
        gd = torch.as_tensor(g.astype(npdt), device="cuda")
        cd = torch.as_tensor(c, device="cuda")
        z = torch.empty_like(gd)
        op.precond_("stencil" if kind == "stencil" else "fft", gd, cd, z, radius=radius)
        torch.cuda.synchronize()
        ref = P.apply(g.astype(npdt), c.astype(bool), npdt).astype(np.float64)
        got = z.cpu().numpy().astype(np.float64)
        assert np.all(got[c == 0] == 0.0)
        assert rel(got, ref) < tol
        assert abs(got[c == 1].astype(np.float64).sum()) <= 1e-5 * np.abs(got).sum()
