"""The allocation-free periodic apply (aspher_periodic_matvec_noalloc).

Some callers of this library cannot let it allocate device memory --
real-time loops that must not block in the allocator, hosts whose own
allocator owns the GPU's memory -- so this entry point keeps its scratch in a
static device array instead.  Its output must match the operator entry point's
(aspher_op_matvec on a periodic operator) within the tolerances the other
operator tests use, on two calls in a row (the second call reuses the
scratch the first one left behind); once set up, calls must leave the
device's free memory unchanged; bad arguments are rejected before any
launch.  This file is collected last.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _noalloc(Ns, L, E, x, y, dtype=None):
    from aspher_b200 import _lib
    if dtype is None:
        dtype = _lib.F64 if x.dtype == torch.float64 else _lib.F32
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    xp = C.c_void_p(x if isinstance(x, int) else x.data_ptr())
    yp = C.c_void_p(y if isinstance(y, int) else y.data_ptr())
    return _lib.lib().aspher_periodic_matvec_noalloc(Ns, L, E, dtype, xp, yp, stream)


@pytest.mark.parametrize("Ns", [16, 256, 1024])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 2e-6)])
def test_noalloc_matches_operator_apply_twice(Ns, dtype, tol):
    from aspher_b200 import Operator
    L, E = 1.7, 0.8
    op = Operator("periodic", Ns, L, E)
    rng = np.random.default_rng(Ns)
    for call in range(2):
        x = torch.as_tensor(rng.standard_normal(Ns * Ns), dtype=dtype, device="cuda")
        ref = torch.empty_like(x)
        op.matvec_(x, ref)
        y = torch.full_like(x, float("nan"))
        assert _noalloc(Ns, L, E, x, y) == 0
        torch.cuda.synchronize()
        a = y.double().cpu().numpy()
        b = ref.double().cpu().numpy()
        assert np.all(np.isfinite(a)), call
        assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b), call


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_calls_leave_device_memory_unchanged(dtype):
    """After a first (set-up) call, steady-state calls allocate nothing: the
    device's free memory (cudaMemGetInfo) is the same before and after."""
    Ns = 1024
    x = torch.randn(Ns * Ns, dtype=dtype, device="cuda")
    y = torch.empty_like(x)
    assert _noalloc(Ns, 1.0, 1.0, x, y) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert _noalloc(Ns, 1.0, 1.0, x, y) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from aspher_b200 import _lib
    x = torch.zeros(2048 * 2048, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    assert _noalloc(2048, 1.0, 1.0, x, y) == _lib.ASPHER_EINVAL
    assert b"[16, 1024]" in _lib.lib().aspher_last_error()
    assert _noalloc(24, 1.0, 1.0, x, y) == _lib.ASPHER_EINVAL


def test_noalloc_rejects_bad_buffers_and_dtype():
    """Misaligned (8-byte offset) and NULL buffers, an unknown dtype and a
    non-positive domain size return ASPHER_EINVAL without launching."""
    from aspher_b200 import _lib
    Ns = 64
    x = torch.zeros(Ns * Ns + 2, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    E = _lib.ASPHER_EINVAL
    assert _noalloc(Ns, 1.0, 1.0, x.data_ptr() + 8, y, dtype=_lib.F64) == E
    assert b"aligned" in _lib.lib().aspher_last_error()
    assert _noalloc(Ns, 1.0, 1.0, x, y.data_ptr() + 8, dtype=_lib.F64) == E
    assert _noalloc(Ns, 1.0, 1.0, 0, y, dtype=_lib.F64) == E
    assert _noalloc(Ns, 1.0, 1.0, x, 0, dtype=_lib.F64) == E
    assert b"NULL" in _lib.lib().aspher_last_error()
    assert _noalloc(Ns, 1.0, 1.0, x, y, dtype=7) == E
    assert b"dtype" in _lib.lib().aspher_last_error()
    assert _noalloc(Ns, 0.0, 1.0, x, y, dtype=_lib.F64) == E
    torch.cuda.synchronize()
