"""The tangential (Cerruti) FFT operator on the device (B200).

Gates (the reference's test_tangential.cpp:25-41 and the oracle):
* equal to the dense block [[XX, XY], [XY, YY]] built from the reference's
  own CerrutiKernel tables (oracle/_ref, else the pinned restatement):
  FP64 rel < 1e-13, FP32 < 1e-5;
* equal to the numpy restatement of TangentialFFTOperator at Ns up to
  2048: FP64 1e-13, FP32 2e-6;
* the device tables equal the reference's; the build's realness check;
* u may alias q; bitwise repeatable; invalid sizes rejected.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import ref  # noqa: E402
from oracle.tangential import CerrutiKernel, TangentialFFTOperator  # noqa: E402

pytestmark = pytest.mark.gpu


def _dense_from_tables(Ns, xx, yy, xy):
    N = Ns * Ns
    i = np.arange(N)
    ix, iy = i % Ns, i // Ns
    dix = ix[:, None] - ix[None, :] + Ns - 1
    diy = iy[:, None] - iy[None, :] + Ns - 1
    return np.block([[xx[diy, dix], xy[diy, dix]], [xy[diy, dix], yy[diy, dix]]])


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize("Ns", [16, 32])
def test_tangential_matches_dense_block(Ns):
    from aspher_b200 import TangentialOperator
    L, E, nu = 1.0, 1.7, 0.3
    op = TangentialOperator(Ns, L, E, nu)
    if ref.available():
        tabs = ref.cerruti_tables(Ns, L, E, nu)
    else:
        C = CerrutiKernel(Ns, L, E, nu)
        d = np.arange(-(Ns - 1), Ns)
        tabs = C.offsets(d[None, :], d[:, None])
    D = _dense_from_tables(Ns, *tabs)
    q = np.random.default_rng(7 + Ns).uniform(-1, 1, 2 * Ns * Ns)
    want = D @ q
    assert _rel(op.matvec(q), want) < 1e-13
    q32 = torch.as_tensor(q, dtype=torch.float32, device="cuda")
    u32 = torch.empty_like(q32)
    op.matvec_(q32, u32)
    assert _rel(u32.double().cpu().numpy(), want) < 1e-5
    assert op.max_im_ratio <= 1e-10


@pytest.mark.parametrize("Ns", [64, 256, 1024, 2048])
def test_tangential_matches_oracle(Ns):
    from aspher_b200 import TangentialOperator
    L, E, nu = 1.3, 0.9, 0.25
    op = TangentialOperator(Ns, L, E, nu)
    F = TangentialFFTOperator(CerrutiKernel(Ns, L, E, nu))
    q = np.random.default_rng(Ns).standard_normal(2 * Ns * Ns)
    want = F.matvec(q)
    assert _rel(op.matvec(q), want) <= 1e-13
    q32 = torch.as_tensor(q, dtype=torch.float32, device="cuda")
    u32 = torch.empty_like(q32)
    op.matvec_(q32, u32)
    assert _rel(u32.double().cpu().numpy(), want) <= 2e-6


def test_tangential_tables_match_reference():
    from aspher_b200 import TangentialOperator
    Ns, L, E, nu = 32, 1.1, 1.7, 0.3
    op = TangentialOperator(Ns, L, E, nu)
    got = op.tables()
    if ref.available():
        want = ref.cerruti_tables(Ns, L, E, nu)
    else:
        C = CerrutiKernel(Ns, L, E, nu)
        d = np.arange(-(Ns - 1), Ns)
        want = C.offsets(d[None, :], d[:, None])
    scale = np.max(np.abs(want[0]))
    for g, w in zip(got, want):
        assert np.max(np.abs(g - w)) <= 1e-14 * scale


def test_tangential_inplace_repeatable_and_rejects():
    from aspher_b200 import TangentialOperator
    Ns = 128
    op = TangentialOperator(Ns)
    q = torch.randn(2 * Ns * Ns, dtype=torch.float64, device="cuda")
    u1 = torch.empty_like(q)
    u2 = torch.empty_like(q)
    op.matvec_(q, u1)
    op.matvec_(q, u2)
    assert torch.equal(u1, u2)
    qi = q.clone()
    op.matvec_(qi, qi)  # u aliases q
    assert torch.equal(qi, u1)
    with pytest.raises(ValueError):
        TangentialOperator(4096)
    with pytest.raises(ValueError):
        TangentialOperator(1)
    with pytest.raises(ValueError):
        TangentialOperator(64, nu=1.0)


def _hertz_threshold(Ns, mu=0.3, a2=0.09):
    """s = mu p on a Hertz-like pressure disk (open points outside)."""
    x = (np.arange(Ns) + 0.5) / Ns - 0.5
    r2 = x[None, :] ** 2 + x[:, None] ** 2
    return mu * np.sqrt(np.maximum(0.0, a2 - r2)).ravel()


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("Ns", [32, 64])
@pytest.mark.parametrize("mode", ["displacement", "force"])
def test_tangential_solve_matches_reference(Ns, mode):
    """solve_tangential (src/friction_solve.cpp:375-688) on the device against
    the reference's own solve on the same operator: the same status, the
    stick / slip partition within a few points, the local KKT residuals at
    the reference's level, force control's mean traction exact.

    Displacement control is a strictly convex problem solved to tol: the
    tractions agree to 1e-6.  Force control stops its outer Newton/Broyden
    iteration at the inner solver's floor (friction_solve.cpp:576-612) and
    closes the load with the terminal correction, so its answer is defined
    only to that floor: the reference's own tractions at tol 1e-8 and 1e-10
    differ by 2.3e-3 (Ns = 32) and its tol 1e-8 and 1e-12 ones by 1.6e-3
    (Ns = 64), and its acceptance (friction_solve.cpp:399-413) is local KKT
    within 1e-2.  The force-control gate is the reference's acceptance
    level: tractions within 1e-2, the rigid shift (the multiplier of
    mean(q) = q_bar, to which the outer iteration's load residual F maps
    through the 2x2 stiffness) within 1e-3 -- the acceptance
    F <= 1e-3 |q_bar| -- and both KKT certificates passing.  The inner
    iteration itself is pinned tightly in
    test_tangential_warm_solve_equals_reference."""
    from aspher_b200 import TangentialOperator
    s = _hertz_threshold(Ns)
    if mode == "displacement":
        fc, target = False, (2e-3, -1e-3)
    else:
        fc, target = True, (0.3 * s.mean(), 0.1 * s.mean())
    qr, dr = ref.Tangential(Ns).solve(s, fc, target, tol=1e-8, max_iter=5000)
    q, d = TangentialOperator(Ns).solve(s, force_control=fc, target=target, tol=1e-8,
                                        max_iter=5000)
    assert dr["status"] == "converged"
    assert d["status"] == "converged", d
    assert _rel(q, qr) <= (1e-2 if fc else 1e-6)
    assert abs(d["n_stick"] - dr["n_stick"]) <= 3 and abs(d["n_slip"] - dr["n_slip"]) <= 3
    assert d["n_open"] == dr["n_open"]
    assert d["cone_violation"] <= 1e-9
    if fc:
        assert d["proj_residual"] <= d["kkt_tol"] and d["force_error"] <= 1e-12
    else:
        assert d["proj_residual"] <= max(10 * dr["proj_residual"], 1e-8)
    if fc:
        assert abs(d["q_mean"][0] - target[0]) <= 1e-12 * abs(target[0])
        assert abs(d["q_mean"][1] - target[1]) <= 1e-12 * abs(target[0])
        assert abs(d["delta_t"][0] - dr["delta_x"]) <= 1e-3 * abs(dr["delta_x"])
        assert abs(d["delta_t"][1] - dr["delta_y"]) <= 1e-3 * abs(dr["delta_x"])
    else:
        assert d["delta_t"] == target


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("Ns", [32, 64])
def test_tangential_warm_solve_equals_reference(Ns):
    """The step force control repeats: a displacement-control solve warm-
    started from the previous traction (friction_solve.cpp:586-590).  From the
    same start the device iteration follows the reference's step by step:
    the same iteration count and tractions equal to 1e-10 (the unpreconditioned
    tangential PCG stalls at a local-KKT floor of 1e-4 .. 1e-3 at this load,
    so cold solves from roundoff-different starts part ways at that level;
    the warm chain does not).

    The reference runs on one OpenMP thread here: its sums are OpenMP
    reductions (friction_solve.cpp:102, 198, 219), which combine the
    threads' partial sums in arrival order, so with three or more threads
    its own trajectory changes from run to run in the last bits, and the
    iteration count of a run that ends on the stall rule with it."""
    from aspher_b200 import TangentialOperator
    s = _hertz_threshold(Ns)
    target = (0.3 * s.mean(), 0.1 * s.mean())
    nt = ref.threads()
    ref.set_threads(1)
    try:
        q0, d0 = ref.Tangential(Ns).solve(s, True, target, tol=1e-8, max_iter=5000)
        delta = (d0["delta_x"] * 1.0001, d0["delta_y"])
        qr, dr = ref.Tangential(Ns).solve(s, False, delta, tol=1e-8, max_iter=5000, q_init=q0)
    finally:
        ref.set_threads(nt)
    q, d = TangentialOperator(Ns).solve(s, force_control=False, target=delta, tol=1e-8,
                                        max_iter=5000, q_init=q0)
    assert d["status"] == dr["status"]
    assert d["iterations"] == dr["iterations"]
    # the transforms' rounding differs from the reference's engine (the
    # first forward stage skips the zero half): 1e-10 after ~200 steps
    assert _rel(q, qr) <= 1e-10


def test_tangential_solve_rejects():
    from aspher_b200 import TangentialOperator
    Ns = 32
    op = TangentialOperator(Ns)
    s = _hertz_threshold(Ns)
    with pytest.raises(ValueError, match="gross-slip"):
        op.solve(s, force_control=True, target=(s.mean(), 0.0))
    with pytest.raises(ValueError, match="negative"):
        op.solve(-s, target=(1e-3, 0.0))
    with pytest.raises(ValueError, match="everywhere"):
        op.solve(np.zeros(Ns * Ns), target=(1e-3, 0.0))


@pytest.mark.parametrize("Ns", [5, 12, 37, 100])
def test_tangential_embedded_grid_matches_reference(Ns):
    """Grids that are not powers of two (the reference's TangentialFFTOperator
    takes any Ns): the caller's block inside the next power of two's
    pipeline, the Cerruti tables at the caller's cell size.  Against the
    dense block of the reference's own tables (FP64 1e-13, FP32 1e-5) and
    the reference's own apply where it is built."""
    from aspher_b200 import TangentialOperator
    L, E, nu = 1.3, 0.9, 0.25
    op = TangentialOperator(Ns, L, E, nu)
    if ref.available():
        tabs = ref.cerruti_tables(Ns, L, E, nu)
    else:
        C = CerrutiKernel(Ns, L, E, nu)
        d = np.arange(-(Ns - 1), Ns)
        tabs = C.offsets(d[None, :], d[:, None])
    got_tabs = op.tables()
    scale = np.max(np.abs(tabs[0]))
    for a, b in zip(got_tabs, tabs):
        assert np.max(np.abs(a - b)) <= 1e-14 * scale
    D = _dense_from_tables(Ns, *tabs)
    q = np.random.default_rng(3 + Ns).uniform(-1, 1, 2 * Ns * Ns)
    want = D @ q
    assert _rel(op.matvec(q), want) < 1e-13
    q32 = torch.as_tensor(q, dtype=torch.float32, device="cuda")
    u32 = torch.empty_like(q32)
    op.matvec_(q32, u32)
    assert _rel(u32.double().cpu().numpy(), want) < 1e-5
    if ref.available():
        assert _rel(op.matvec(q), ref.Tangential(Ns, L, E, nu).matvec(q)) < 1e-13


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("mode", ["displacement", "force"])
def test_tangential_embedded_solve_matches_reference(mode):
    """solve_tangential on a 40 x 40 grid (embedded in 64): the cells outside
    the caller's block are open (s = 0), the mean traction and the cell
    counts are the caller's.  Displacement control: traction to 1e-6; force
    control: at the reference's acceptance (see
    test_tangential_solve_matches_reference); the warm chain step by step."""
    from aspher_b200 import TangentialOperator
    Ns = 40
    s = _hertz_threshold(Ns)
    op = TangentialOperator(Ns)
    if mode == "displacement":
        fc, target = False, (2e-3, -1e-3)
    else:
        fc, target = True, (0.3 * s.mean(), 0.1 * s.mean())
    qr, dr = ref.Tangential(Ns).solve(s, fc, target, tol=1e-8, max_iter=5000)
    q, d = op.solve(s, force_control=fc, target=target, tol=1e-8, max_iter=5000)
    assert q.shape == (2 * Ns * Ns,)
    assert dr["status"] == "converged" and d["status"] == "converged", d
    assert d["n_stick"] + d["n_slip"] + d["n_open"] == Ns * Ns
    assert d["n_open"] == dr["n_open"]
    assert abs(d["n_stick"] - dr["n_stick"]) <= 3
    assert d["cone_violation"] <= 1e-9 and d["proj_residual"] <= d["kkt_tol"]
    assert abs(d["w_ref"] - dr["w_ref"]) <= 1e-12 * dr["w_ref"]
    if fc:
        assert _rel(q, qr) <= 1e-2
        assert abs(d["q_mean"][0] - target[0]) <= 1e-12 * abs(target[0])
        assert abs(d["delta_t"][0] - dr["delta_x"]) <= 1e-3 * abs(dr["delta_x"])
    else:
        assert _rel(q, qr) <= 1e-6
        delta = (target[0] * 1.0001, target[1])
        qr2, dr2 = ref.Tangential(Ns).solve(s, False, delta, tol=1e-8, max_iter=5000, q_init=qr)
        q2, d2 = op.solve(s, force_control=False, target=delta, tol=1e-8, max_iter=5000,
                          q_init=qr)
        # the embedded transform (64-point pipeline against the reference's
        # 80-point one) rounds differently: the chain may stop one step
        # apart, its tractions within the tolerance's reach
        assert abs(d2["iterations"] - dr2["iterations"]) <= 1
        assert _rel(q2, qr2) <= 1e-7
