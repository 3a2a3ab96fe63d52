"""Launch variants of the FFT passes (B200).

Every (row, column) launch-variant pair of an operator gives the same apply
up to the rounding of its transform shape: a variant change re-tiles the
half spectrum for the column tile width it implies, and with it the
free-space Kh and the periodic multiplier table, and switches the row
passes between their fixed-stride and general tile forms.  The autotuner
leaves the apply unchanged the same way.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _apply(op, x):
    y = torch.empty_like(x)
    op.matvec_(x, y)
    torch.cuda.synchronize()
    return y.double().cpu().numpy()


@pytest.mark.parametrize("backend", ["fft", "periodic"])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 2e-6)])
@pytest.mark.parametrize("Ns", [256, 1024])
def test_every_variant_pair_gives_the_same_apply(backend, dtype, tol, Ns):
    import aspher_b200 as asb
    op = asb.Operator(backend, Ns)
    rv0, cv0, _ = op.variants(dtype)
    g = torch.Generator(device="cuda")
    g.manual_seed(Ns)
    x = torch.randn(Ns * Ns, dtype=dtype, device="cuda", generator=g)
    y0 = _apply(op, x)
    n0 = np.linalg.norm(y0)
    widths = set()
    for rv in range(4):
        for cv in range(4):
            op.set_variants(rv, cv, dtype)
            assert op.variants(dtype)[:2] == (rv, cv)
            widths.add(op.variants(dtype)[2])
            y = _apply(op, x)
            assert np.linalg.norm(y - y0) <= tol * n0, (rv, cv)
    # the sweep crossed column tile widths (so the tables were re-tiled)
    assert len(widths) > 1
    op.set_variants(rv0, cv0, dtype)
    assert np.array_equal(_apply(op, x), y0)


@pytest.mark.parametrize("backend", ["fft", "periodic"])
def test_autotune_keeps_the_apply(backend):
    import aspher_b200 as asb
    Ns = 512
    op = asb.Operator(backend, Ns)
    x = torch.randn(Ns * Ns, dtype=torch.float32, device="cuda")
    y0 = _apply(op, x)
    rv, cv, ms = op.autotune(torch.float32, reps=2)
    assert 0 <= rv < 4 and 0 <= cv < 4 and ms > 0.0
    assert op.variants(torch.float32)[:2] == (rv, cv)
    y = _apply(op, x)
    assert np.linalg.norm(y - y0) <= 2e-6 * np.linalg.norm(y0)
