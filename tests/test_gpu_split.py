"""Split transforms and the largest grids (B200).

The zero-padded free-space column of length 2 Ns is transformed as two
length-Ns halves (even and odd frequencies).  That is the only form an FP64
column of 16384 points can take (it does not fit one CTA's shared memory), so
FP64 applies at Ns = 8192 and FP32 applies at Ns = 16384 use it; the
operator creation flag SPLIT_COLUMNS forces it at smaller sizes, where it is checked
against the oracle and against the one-CTA column pass.  The FP64 Kh build
likewise assembles rows of 2 Ns reals from the transforms of their even and
odd samples where a row does not fit (Ns = 16384); the flag SPLIT_KH forces
that form for the cross-check.  Applies at the large sizes are checked
through point loads, whose response is the Love table itself (the aperiodic
convolution of a unit load at a corner cell), through exact periodic Fourier
modes, against the other precision, and for symmetry.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle.operators import FFTOperator as OFFT  # noqa: E402

pytestmark = pytest.mark.gpu


def _op(Ns, split=False, flag="SPLIT_COLUMNS", backend="fft"):
    from aspher_b200 import Operator
    return Operator(backend, Ns, flags=getattr(Operator, flag) if split else 0)


def _mv(op, x, dtype):
    xt = torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device="cuda")
    y = torch.empty_like(xt)
    op.matvec_(xt, y)
    torch.cuda.synchronize()
    return y.cpu().numpy().astype(np.float64)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("Ns", [256, 1024])
def test_split_columns_match_oracle_and_one_cta_form(Ns):
    ops, op = _op(Ns, split=True), _op(Ns)
    x = np.random.default_rng(11).standard_normal(Ns * Ns)
    ref = OFFT(Ns, 1.0, 1.0).matvec(x)
    ys = _mv(ops, x, torch.float64)
    assert rel(ys, ref) < 1e-13
    assert rel(ys, _mv(op, x, torch.float64)) < 1e-14
    x32 = x.astype(np.float32)
    ref32 = OFFT(Ns, 1.0, 1.0).matvec(x32.astype(np.float64))
    ys32 = _mv(ops, x32, torch.float32)
    assert rel(ys32, ref32) < 2e-6
    # repeat calls bitwise equal (test_fft.cpp:46-59)
    assert np.array_equal(ys, _mv(ops, x, torch.float64))


def test_split_columns_batched_solve():
    import aspher_b200 as asb
    from aspher_b200.surfaces import self_affine_gap
    Ns = 256
    ops, op = _op(Ns, split=True), _op(Ns)
    gs = [torch.from_numpy(self_affine_gap(Ns, hurst=0.8, rms=0.002, seed=s)).cuda()
          for s in (3, 4, 5)]
    loads = [0.002, 0.005, 0.02]
    rb = asb.solve_device_batch(ops, gs, loads, tol=1e-10, precond="fourier",
                                dtype=torch.float64)
    for g, p, r in zip(gs, loads, rb):
        r1 = asb.solve_device(op, g, p, tol=1e-10, precond="fourier", dtype=torch.float64,
                              light=True)
        assert r.status == "converged" and r1.status == "converged"
        assert rel(r.pressure.ravel(), r1.pressure.ravel()) < 1e-8
        assert abs(r.contact_area - r1.contact_area) <= 1e-4


def test_fp64_apply_at_8192():
    Ns = 8192
    N = Ns * Ns
    op = _op(Ns)
    T = op.love_table()
    # unit loads at the two opposite corners: u(iy, ix) = T(|iy - jy|, |ix - jx|)
    for (jy, jx) in ((0, 0), (Ns - 1, Ns - 1)):
        x = np.zeros(N)
        x[jy * Ns + jx] = 1.0
        u = _mv(op, x, torch.float64).reshape(Ns, Ns)
        ref = T if jy == 0 else T[::-1, ::-1]
        assert rel(u.ravel(), ref.ravel()) < 1e-13
        assert np.max(np.abs(u - ref)) < 1e-13 * T[0, 0]
    del T
    rng = np.random.default_rng(5)
    x, w = rng.standard_normal(N), rng.standard_normal(N)
    y = _mv(op, x, torch.float64)
    assert rel(y, _mv(op, x.astype(np.float32), torch.float32)) < 2e-6
    sx, sw = np.dot(w, y), np.dot(x, _mv(op, w, torch.float64))
    assert abs(sx - sw) < 1e-12 * np.linalg.norm(y) * np.linalg.norm(w)


def test_fp64_solve_runs_at_8192():
    import aspher_b200 as asb
    from aspher_b200.surfaces import self_affine_gap
    Ns = 8192
    op = _op(Ns)
    g = torch.from_numpy(self_affine_gap(Ns, hurst=0.8, rms=0.002, seed=42)).cuda()
    r = asb.solve_device(op, g, 0.005, tol=1e-6, max_iter=8, precond="fourier",
                         dtype=torch.float64, light=True)
    assert r.iterations == 8 and r.status == "max_iterations"
    p = r.pressure_device
    assert torch.isfinite(p).all() and float(p.min()) >= 0.0
    assert abs(float(p.mean()) / 0.005 - 1.0) < 1e-12


@pytest.mark.parametrize("Ns", [256, 1024])
def test_split_kh_build_matches_one_cta_build(Ns):
    opk, op = _op(Ns, split=True, flag="SPLIT_KH"), _op(Ns)
    assert opk.info().max_im_ratio < 1e-10
    x = np.random.default_rng(13).standard_normal(Ns * Ns)
    y = _mv(op, x, torch.float64)
    assert rel(_mv(opk, x, torch.float64), y) < 1e-14
    assert rel(y, OFFT(Ns, 1.0, 1.0).matvec(x)) < 1e-13


def test_fp32_free_space_at_16384():
    Ns = 16384
    N = Ns * Ns
    op = _op(Ns)
    assert op.info().max_im_ratio < 1e-10
    T = op.love_table()
    for (jy, jx) in ((0, 0), (Ns - 1, Ns - 1)):
        x = torch.zeros(N, dtype=torch.float32, device="cuda")
        x[jy * Ns + jx] = 1.0
        y = torch.empty_like(x)
        op.matvec_(x, y)
        u = y.double().cpu().numpy().reshape(Ns, Ns)
        ref = T if jy == 0 else T[::-1, ::-1]
        assert rel(u.ravel(), ref.ravel()) < 2e-6
        assert np.max(np.abs(u - ref)) < 2e-6 * T[0, 0]
        del u
    del T
    with pytest.raises(Exception):
        x = torch.zeros(N, dtype=torch.float64, device="cuda")
        op.matvec_(x, torch.empty_like(x))
    torch.cuda.synchronize()


def test_fp32_periodic_modes_at_16384():
    Ns, L, Es = 16384, 3.0, 2.5
    from aspher_b200 import Operator
    op = Operator("periodic", Ns, L, Es)
    ix = torch.arange(Ns, dtype=torch.float64, device="cuda")
    for mx, my in ((1, 0), (3, 7), (4000, 123)):
        q = 2 * np.pi * np.hypot(mx, my) / L
        p = torch.cos(2 * np.pi * ((mx * ix[None, :] + my * ix[:, None]) % Ns) / Ns)
        p32 = p.float().reshape(-1).contiguous()
        y = torch.empty_like(p32)
        op.matvec_(p32, y)
        ref = (2.0 / (Es * q)) * p32.double()
        assert float(torch.linalg.norm(y.double() - ref) / torch.linalg.norm(ref)) < 2e-6
        del p, p32, y, ref
    torch.cuda.synchronize()


def test_fp32_solves_at_16384():
    import aspher_b200 as asb
    Ns = 16384
    # a wavy surface made on the device (a 16384^2 self-affine field would take
    # tens of GB of host memory to synthesise)
    x = torch.arange(Ns, dtype=torch.float64, device="cuda") / Ns
    g = (-0.001 * (torch.cos(2 * np.pi * 3 * x)[None, :] + torch.cos(2 * np.pi * 5 * x)[:, None]
                   + 0.3 * torch.sin(2 * np.pi * 17 * (x[None, :] + 2 * x[:, None])))).reshape(-1)
    for backend in ("fft", "periodic"):
        op = _op(Ns, backend=backend)
        r = asb.solve_device(op, g, 0.005, tol=1e-6, max_iter=6, precond="fourier",
                             dtype=torch.float32, light=True)
        assert r.iterations == 6 and r.status == "max_iterations"
        p = r.pressure_device
        assert torch.isfinite(p).all() and float(p.min()) >= 0.0
        assert abs(float(p.double().mean()) / 0.005 - 1.0) < 1e-6
        del op, r, p
        torch.cuda.empty_cache()


def test_fp32_nested_at_16384_and_fp64_rejected():
    """solve_nested up to Ns = 16384 in FP32 (the size at which the
    reference's fft rows ran out of memory); FP64 there is refused with
    ValueError."""
    import aspher_b200 as asb
    from aspher_b200.surfaces import self_affine_gap_device
    Ns, pbar = 16384, 0.002
    g = self_affine_gap_device(Ns, hurst=0.8, rms=0.02, k_lo=12.0, k_hi=0.33 * Ns, seed=42)
    r = asb.solve_nested(Ns, g, pbar, coarsest=4096, tol=1e-6, single_precision=True,
                         allow_tolerance_relaxation=True, light_result=True, backend="fft")
    assert r.status == "converged", (r.status, r.status_reason)
    assert [st["name"] for st in r.stage_stats] == ["coarse:4096", "coarse:8192",
                                                    "finest:16384"]
    assert r.fw_error <= r.effective_tol and r.penetration_error <= r.effective_tol
    p = r.pressure_device
    assert float(p.min()) >= 0.0 and abs(float(p.mean()) / pbar - 1.0) < 1e-6
    assert 0.0 < r.contact_area < 0.05
    del p, r
    torch.cuda.empty_cache()
    with pytest.raises(ValueError):
        asb.solve_nested(Ns, g, pbar, coarsest=8192, tol=1e-6, light_result=True,
                         backend="fft", precision="double")
