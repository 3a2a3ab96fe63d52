"""Pins of the tangential (Cerruti) oracle (CPU).

* the Cerruti brackets against the reference's 80-digit fixture
  (tests/data/cerruti_reference.txt, committed as
  tests/golden/cerruti_reference.txt; the reference's gate in
  test_kernel_stability.cpp:215-262: 1e-12 against max(|value|, the local
  Love scale));
* the identities of test_cerruti.cpp:80-140 (nu = 0 is Love, parities,
  self terms, signed-offset symmetry);
* the kernel tables against the reference's own CerrutiKernel
  (oracle/_ref, src/cerruti_kernel.cpp) to rounding;
* the FFT operator against the dense block matrix [[XX, XY], [XY, YY]]
  (test_tangential.cpp:25-41: rel < 1e-13).
"""

import os

import numpy as np
import pytest

from oracle import ref
from oracle.love import love_uz
from oracle.tangential import (CerrutiKernel, TangentialFFTOperator, cerruti_uxx,
                               cerruti_uxy)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_cerruti_brackets_vs_reference_fixture():
    r = np.loadtxt(os.path.join(GOLDEN, "cerruti_reference.txt"))
    assert len(r) == 58
    x, y, a, b, ylog, uxy = r.T
    got_ylog = cerruti_uxx(x, y, a, b, 1.0)  # nu = 1 isolates ylog
    got_uxy = cerruti_uxy(x, y, a, b)
    scale = love_uz(x, y, a, b)
    e1 = np.abs(got_ylog - ylog) / np.maximum(np.abs(ylog), scale)
    e2 = np.abs(got_uxy - uxy) / np.maximum(np.abs(uxy), scale)
    assert e1.max() <= 1e-12 and e2.max() <= 1e-12


def test_cerruti_identities():
    """test_cerruti.cpp:80-100."""
    a, b, x, y, nu = 0.011, 0.017, 0.05, -0.03, 0.31
    assert abs(cerruti_uxx(x, y, a, b, 0.0) / love_uz(x, y, a, b) - 1.0) < 1e-13
    assert cerruti_uxx(x, y, a, b, nu) == cerruti_uxx(-x, y, a, b, nu)
    assert cerruti_uxx(x, y, a, b, nu) == cerruti_uxx(x, -y, a, b, nu)
    assert cerruti_uxy(-x, y, a, b) == -cerruti_uxy(x, y, a, b)
    assert cerruti_uxy(x, -y, a, b) == -cerruti_uxy(x, y, a, b)
    self = (2.0 - nu) * 4.0 * a * np.log(1.0 + np.sqrt(2.0))
    assert abs(cerruti_uxx(0.0, 0.0, a, a, nu) / self - 1.0) < 1e-14
    assert cerruti_uxy(0.0, 0.0, a, a) == 0.0


def test_cerruti_kernel_offsets():
    """test_cerruti.cpp:102-140 (signed offsets, self term, symmetric dense)."""
    Ns, L, E, nu = 16, 1.0, 1.7, 0.3
    C = CerrutiKernel(Ns, L, E, nu)
    a = 0.5 * L / Ns
    self = (2.0 - nu) * 4.0 * a * np.log(1.0 + np.sqrt(2.0)) / (np.pi * E * (1.0 - nu))
    xx, yy, xy = C.offsets(np.array([0, 3, -3, 2, -2, 2, 0, 4, Ns]),
                           np.array([0, 1, 1, 5, 5, -5, 4, 0, 0]))
    assert abs(xx[0] / self - 1.0) < 1e-14 and xy[0] == 0.0
    assert yy[1] == C.offsets(1, 3)[0]
    assert xx[2] == xx[1]
    assert xy[3] == C.offsets(-2, -5)[2]
    assert xy[4] == -xy[3] and xy[5] == -xy[3]
    assert xy[6] == 0.0 and xy[7] == 0.0 and xx[8] == 0.0
    D = C.assemble_dense()
    assert np.max(np.abs(D - D.T)) == 0.0
    np.linalg.cholesky(D)  # positive definite (elastic compliance)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("Ns", [8, 24])
def test_cerruti_tables_match_reference(Ns):
    """The oracle's tables against the reference's CerrutiKernel itself."""
    L, E, nu = 1.3, 1.7, 0.3
    rx, ryy, rxy = ref.cerruti_tables(Ns, L, E, nu)
    C = CerrutiKernel(Ns, L, E, nu)
    d = np.arange(-(Ns - 1), Ns)
    xx, yy, xy = C.offsets(d[None, :], d[:, None])
    scale = np.max(np.abs(rx))
    assert np.max(np.abs(xx - rx)) <= 1e-14 * scale
    assert np.max(np.abs(yy - ryy)) <= 1e-14 * scale
    assert np.max(np.abs(xy - rxy)) <= 1e-14 * scale


@pytest.mark.parametrize("Ns", [8, 16])
def test_tangential_fft_matches_dense(Ns):
    """test_tangential.cpp:25-41: the FFT operator reproduces the dense
    Cerruti block to roundoff; FP32 to 1e-5."""
    C = CerrutiKernel(Ns, 1.0, 1.7, 0.3)
    F = TangentialFFTOperator(C)
    D = C.assemble_dense()
    q = np.random.default_rng(7 + Ns).uniform(-1, 1, 2 * Ns * Ns)
    want = D @ q
    got = F.matvec(q)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-13
    got32 = F.matvec(q.astype(np.float32), np.float32).astype(np.float64)
    assert np.linalg.norm(got32 - want) / np.linalg.norm(want) < 1e-5
