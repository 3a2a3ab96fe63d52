"""Batched solves (one loop graph for several problems on one operator).

Each problem of a batch must come out as the single-problem solve of the
same inputs: the kernels are the same, instance b reads only its own
parameters, state, partials and fields, and its reductions run on the same
grid in the same order, so FP64 results agree to reduction-order roundoff
and iteration counts are equal.  Problems that halt early (converged,
max_iterations, or a host-side identification step) must not disturb the
others (the per-instance convergence masks).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _rough(Ns, seed):
    from aspher_b200 import self_affine_gap
    return self_affine_gap(Ns, hurst=0.8, rms=0.002, k_lo=2.0, k_hi=Ns / 4, seed=seed)


def rel(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_batch_equals_single(backend, dtype):
    from aspher_b200 import Operator, solve_device, solve_device_batch
    Ns = 64
    op = Operator(backend, Ns)
    loads = [0.002, 0.01, 0.03]
    gaps = [torch.as_tensor(_rough(Ns, 40 + i), device="cuda").to(dtype) for i in range(3)]
    tol = 1e-8 if dtype == torch.float64 else 1e-5
    rb = solve_device_batch(op, gaps, loads, tol=tol, precond="fourier", dtype=dtype)
    for g, pn, r in zip(gaps, loads, rb):
        r1 = solve_device(op, g, pn, tol=tol, precond="fourier", dtype=dtype, light=True,
                          keep_best=True)
        assert r.status == r1.status == "converged"
        assert r.iterations == r1.iterations
        assert rel(r.pressure, r1.pressure) <= (1e-12 if dtype == torch.float64 else 1e-6)
        assert abs(r.contact_area - r1.contact_area) <= 1e-12


@pytest.mark.parametrize("loads", [[0.03, 0.002, 0.01, 0.03], [0.002, 0.03, 0.03, 0.01]])
def test_batch_any_halting_order(loads):
    """The loop graph covers the smallest instance range holding every
    running instance, and shrinks it as end instances halt: instances that
    halt in the middle of the range, at its ends, or in either order keep
    the single-solve results."""
    from aspher_b200 import Operator, solve_device, solve_device_batch
    Ns = 64
    op = Operator("periodic", Ns)
    gaps = [torch.as_tensor(_rough(Ns, 60 + i), device="cuda") for i in range(len(loads))]
    rb = solve_device_batch(op, gaps, loads, tol=1e-9, precond="fourier")
    its = []
    for g, pn, r in zip(gaps, loads, rb):
        r1 = solve_device(op, g, pn, tol=1e-9, precond="fourier", light=True, keep_best=True)
        assert r.status == r1.status == "converged"
        assert r.iterations == r1.iterations
        assert rel(r.pressure, r1.pressure) <= 1e-12
        its.append(r.iterations)
    assert len(set(its)) > 1  # the instances do halt at different iterations


def test_batch_with_identification_and_maxiter():
    from aspher_b200 import Operator, solve_device, solve_device_batch
    Ns = 16
    x = (np.arange(Ns) + 0.5) / Ns - 0.5
    hertz = torch.as_tensor((x[:, None] ** 2 + x[None, :] ** 2).ravel(), device="cuda")
    rough = torch.as_tensor(_rough(Ns, 7), device="cuda")
    op = Operator("fft", Ns)
    warm = torch.zeros(Ns * Ns, dtype=torch.float64, device="cuda")
    warm[0] = 0.01 * Ns * Ns  # singleton warm start: |C| < 2 -> identification step
    rb = solve_device_batch(op, [hertz, rough, hertz], [0.01, 0.005, 0.01], tol=1e-10,
                            precond="none", p_inits=[warm, None, None])
    singles = [solve_device(op, hertz, 0.01, tol=1e-10, p_init=warm, light=True,
                            keep_best=True),
               solve_device(op, rough, 0.005, tol=1e-10, light=True, keep_best=True),
               solve_device(op, hertz, 0.01, tol=1e-10, light=True, keep_best=True)]
    for r, r1 in zip(rb, singles):
        assert r.status == r1.status == "converged"
        assert r.iterations == r1.iterations
        assert r.identification_steps == r1.identification_steps
        assert rel(r.pressure, r1.pressure) <= 1e-12
    assert rb[0].identification_steps >= 1
    # a batch where one problem runs out of iterations and the other converges
    rc = solve_device_batch(op, [hertz, rough], [0.01, 0.005], tol=1e-10, max_iter=3,
                            precond="none")
    r3 = [solve_device(op, g, pn, tol=1e-10, max_iter=3, light=True, keep_best=True)
          for g, pn in ((hertz, 0.01), (rough, 0.005))]
    for r, r1 in zip(rc, r3):
        assert r.status == r1.status
        assert r.iterations == r1.iterations <= 3
        assert rel(r.pressure, r1.pressure) <= 1e-12


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_batch_mixed_matches_single_mixed(backend):
    from aspher_b200 import Operator, solve_device_batch_mixed, solve_device_mixed
    Ns = 128
    op = Operator(backend, Ns)
    loads = [0.003, 0.02]
    gaps = [torch.as_tensor(_rough(Ns, 60 + i), device="cuda") for i in range(2)]
    rb, rbf = solve_device_batch_mixed(op, gaps, loads, tol=1e-6, polish_tol=1e-7,
                                       keep_best=True)
    for g, pn, r, rf in zip(gaps, loads, rb, rbf):
        r1, rf1 = solve_device_mixed(op, g, pn, tol=1e-6, polish_tol=1e-7, light=True,
                                     keep_best=True)
        assert r.status == r1.status == "converged"
        assert rf.iterations == rf1.iterations
        assert r.iterations == r1.iterations
        assert rel(r.pressure, r1.pressure) <= 1e-9
        assert r.requested_tol == 1e-6 and r.fw_error <= 1e-7
