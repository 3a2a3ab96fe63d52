"""Drop-in ``ContactSolver`` / ``solve_nested`` / ``ContactResult`` for the
fft and periodic backends, running on the B200 through libaspher_b200.so.

Mirrors the pybind11 surface of the reference (python/bindings.cpp:115-234
``PyContactSolver``, :362-432 ``py_solve_nested``, :637-879 the module defs):
same argument names, defaults, result fields and errors (ValueError for
invalid input, a status string for numerical outcomes).  PyTorch provides
the device memory and the current CUDA stream; all arithmetic runs in the
library's sm_100a kernels.
"""

import ctypes as C
import time

import numpy as np
import torch

from . import _lib as L


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev():
    if not torch.cuda.is_available():
        raise RuntimeError("aspher_b200 needs a CUDA device (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _to_device_f64(a, expected, dev):
    """numpy array or torch tensor (host, pinned host or device) -> FP64
    device vector of `expected` entries (host->device copy on the current
    stream; non-blocking from pinned memory)."""
    if isinstance(a, torch.Tensor):
        if a.numel() != expected:
            raise ValueError("array has %d entries, expected %d" % (a.numel(), expected))
        t = a.reshape(-1)
        if t.dtype != torch.float64:
            t = t.to(torch.float64)
        return t.to(dev, non_blocking=True)
    return torch.from_numpy(_as_vector(a, expected)).to(dev)


def _as_vector(a, expected, name="array"):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64)).reshape(-1)
    if a.size != expected:
        raise ValueError("%s has %d entries, expected %d" % (name, a.size, expected))
    return a


class Operator:
    """Device operator handle (free-space FFT or periodic)."""

    # creation flags (aspher_op_create_ex): the split column pass and the
    # split FP64 Kh build at sizes where the one-CTA forms fit, for
    # cross-checks of the forms the largest grids need
    SPLIT_COLUMNS = 1
    SPLIT_KH = 2

    def __init__(self, backend, grid_size, domain_size=1.0, E_star=1.0, flags=0):
        if backend not in L.BACKEND:
            raise ValueError("unknown backend: %s (this build implements 'fft' and "
                             "'periodic')" % backend)
        _dev()
        self.backend = backend
        self.Ns = int(grid_size)
        self.N = self.Ns * self.Ns
        self.domain_size = float(domain_size)
        self.E_star = float(E_star)
        h = C.c_void_p()
        L.check(L.lib().aspher_op_create_ex(L.BACKEND[backend], self.Ns, self.domain_size,
                                            self.E_star, int(flags), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().aspher_op_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def matvec_(self, x, y):
        """y = S x on device tensors (float32 or float64, Ns*Ns, contiguous)."""
        dt = L.F64 if x.dtype == torch.float64 else L.F32
        if x.dtype not in (torch.float32, torch.float64) or y.dtype != x.dtype:
            raise ValueError("matvec: float32/float64 tensors of one dtype expected")
        if x.numel() != self.N or y.numel() != self.N:
            raise ValueError("matvec: x size != Ns*Ns")
        if not (x.is_contiguous() and y.is_contiguous()):
            raise ValueError("matvec: contiguous tensors expected")
        L.check(L.lib().aspher_op_matvec(self._h, dt, _ptr(x), _ptr(y), _stream()))
        return y

    def info(self):
        inf = L.OpInfo()
        L.check(L.lib().aspher_op_get_info(self._h, C.byref(inf)))
        return inf

    def variants(self, dtype=torch.float32):
        """(row variant, column variant, column tile width) of this precision."""
        rv, cv, ct = C.c_int(), C.c_int(), C.c_int()
        L.check(L.lib().aspher_op_get_variants(self._h, L.F64 if dtype == torch.float64 else L.F32,
                                               C.byref(rv), C.byref(cv), C.byref(ct)))
        return rv.value, cv.value, ct.value

    def set_variants(self, row_variant, col_variant, dtype=torch.float32):
        L.check(L.lib().aspher_op_set_variants(
            self._h, L.F64 if dtype == torch.float64 else L.F32, int(row_variant),
            int(col_variant)))

    def autotune(self, dtype=torch.float32, reps=5):
        """Time every launch-variant pair of the three FFT passes, keep the
        fastest (also for later operators of this shape); returns
        (row variant, column variant, ms per apply)."""
        rv, cv, ms = C.c_int(), C.c_int(), C.c_double()
        L.check(L.lib().aspher_op_autotune(self._h, L.F64 if dtype == torch.float64 else L.F32,
                                           int(reps), C.byref(rv), C.byref(cv), C.byref(ms)))
        return rv.value, cv.value, ms.value

    def love_table(self):
        out = np.empty((self.Ns, self.Ns), dtype=np.float64)
        L.check(L.lib().aspher_op_love_table(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def precond_(self, precond, g, contact, z, radius=2):
        dt = L.F64 if g.dtype == torch.float64 else L.F32
        L.check(L.lib().aspher_precond_apply(self._h, L.PRECOND[precond], int(radius), dt,
                                             _ptr(g), _ptr(contact), _ptr(z), _stream()))
        return z


def stencil_taps(grid_size, radius=2):
    cap = 64
    dx = (C.c_int * cap)()
    dy = (C.c_int * cap)()
    w = (C.c_double * cap)()
    n = C.c_int()
    L.check(L.lib().aspher_stencil_taps(int(grid_size), int(radius), dx, dy, w, cap,
                                        C.byref(n)))
    return list(dx[:n.value]), list(dy[:n.value]), list(w[:n.value])


class ContactResult:
    """Fields of the reference ``ContactResult`` (bindings.cpp:637-802)."""

    def __init__(self, res, Ns, pressure, displacement=None, gap=None, history=None):
        self._r = res
        self.Ns = Ns
        self._p = pressure
        self._u = displacement
        self._g = gap
        self.error_history = np.asarray(history if history is not None else [], np.float64)
        self.stage_stats = []
        self.time_build = 0.0
        self.time_coarse = 0.0
        self.active_rounds = 0
        self.active_fallback = False
        # accuracy of a float / float_then_double result against the plain
        # FP64 solve of the same problem (ContactSolver.solve(...,
        # reference_fp64=True)); None where it was not measured
        self.pressure_rel_l2_vs_fp64 = None
        self.contact_area_error_vs_fp64 = None
        self.fp64_status = None

    def _grid(self, t):
        if t is None:
            return None
        if isinstance(t, torch.Tensor):
            return t.detach().to("cpu").numpy().reshape(self.Ns, self.Ns)
        return np.asarray(t).reshape(self.Ns, self.Ns)

    @property
    def pressure(self):
        return self._grid(self._p)

    @property
    def pressure_device(self):
        return self._p

    @property
    def displacement(self):
        return self._grid(self._u)

    @property
    def gap(self):
        return self._grid(self._g)

    status = property(lambda s: L.STATUS_NAMES[s._r.status]
                      if 0 <= s._r.status < len(L.STATUS_NAMES) else "unknown")
    status_reason = property(lambda s: s._r.status_reason.decode())
    iterations = property(lambda s: s._r.iterations)
    converged = property(lambda s: bool(s._r.converged))
    contact_area = property(lambda s: s._r.contact_fraction)
    contact_fraction = property(lambda s: s._r.contact_fraction)
    mean_pressure = property(lambda s: s._r.mean_pressure)
    approach = property(lambda s: s._r.approach)
    objective = property(lambda s: s._r.objective)
    error = property(lambda s: s._r.error)
    pk_error = property(lambda s: s._r.pk_error)
    fw_gap = property(lambda s: s._r.fw_gap)
    fw_error = property(lambda s: s._r.fw_error)
    load_error = property(lambda s: s._r.load_error)
    pressure_violation = property(lambda s: s._r.pressure_violation)
    penetration_error = property(lambda s: s._r.penetration_error)
    requested_tol = property(lambda s: s._r.requested_tol)
    effective_tol = property(lambda s: s._r.effective_tol)
    p_ref = property(lambda s: s._r.p_ref)
    g_ref = property(lambda s: s._r.g_ref)
    matvec_count = property(lambda s: s._r.matvec_count)
    verification_matvec_count = property(lambda s: 0)
    precond_count = property(lambda s: s._r.precond_count)
    identification_steps = property(lambda s: s._r.identification_steps)
    returned_best = property(lambda s: bool(s._r.returned_best))
    precond_dropped = property(lambda s: False)
    validation_scope = property(lambda s: "solve_operator")
    operator_error_kind = property(lambda s: "unavailable")
    operator_error = property(lambda s: None)
    objective_error_bound = property(lambda s: None)

    @property
    def memory(self):
        r = self._r
        return dict(cg_state=r.mem_cg_state, best_iterate=r.mem_best_iterate,
                    contact_mask=r.mem_contact_mask, output_arrays=r.mem_output_arrays,
                    peak=r.mem_peak)

    @property
    def timings(self):
        return dict(total=self._r.time_total, matvec=0.0, precond=0.0, build=self.time_build,
                    coarse=self.time_coarse, verification=0.0, candidate=0.0, output=0.0)

    def __repr__(self):
        return ("<ContactResult: %s in %d iters, fw_error %g, penetration %g, contact area %g,"
                " mean p %g>" % (self.status, self.iterations, self.fw_error,
                                 self.penetration_error, self.contact_area,
                                 self.mean_pressure))


def solve_device(op, g0, p_nominal, tol=1e-8, max_iter=5000, use_pr=True, precond="none",
                 p_init=None, dtype=torch.float64, light=False, record_history=False,
                 keep_best=None, requested_tol=0.0, allow_tolerance_relaxation=False,
                 g_ref=0.0, p_ref=0.0, datum_mode="automatic", datum=0.0, precond_radius=2,
                 load_tol=0.0, stall_limit=200, pressure_out=None, loop_mode="graph"):
    """solve_contact_impl<Real> on device tensors (Real = dtype).

    g0 / p_init: device tensors of ``dtype`` (Ns*Ns); the FP64 pressure is
    written to ``pressure_out`` (allocated when None) and stays on the device.
    loop_mode: "graph" (the iterations in a CUDA-graph while loop) or
    "eager" (the same kernels launched one by one, for per-kernel
    profilers; same results, slower).
    """
    N = op.N
    if g0.numel() != N:
        raise ValueError("array has %d entries, expected %d" % (g0.numel(), N))
    if precond not in L.PRECOND:
        raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
    dev = g0.device
    g0 = g0.to(dtype).contiguous()
    if p_init is not None:
        p_init = p_init.to(device=dev, dtype=dtype).contiguous().reshape(-1)
        if p_init.numel() != N:
            raise ValueError("solve_contact: p_init size mismatch")
    o = L.SolveOpts()
    L.lib().aspher_solve_opts_default(C.byref(o))
    o.tol = float(tol)
    o.requested_tol = float(requested_tol)
    o.max_iter = int(max_iter)
    o.use_pr = int(bool(use_pr))
    o.light = int(bool(light))
    o.record_history = int(bool(record_history))
    o.keep_best = int(not light) if keep_best is None else int(bool(keep_best))
    o.load_tol = float(load_tol)
    o.stall_limit = int(stall_limit)
    o.allow_tolerance_relaxation = int(bool(allow_tolerance_relaxation))
    o.precond = L.PRECOND[precond]
    o.precond_radius = int(precond_radius)
    o.p_ref = float(p_ref)
    o.g_ref = float(g_ref)
    o.datum_mode = L.DATUM[datum_mode]
    o.datum = float(datum)
    o.dtype = L.F64 if dtype == torch.float64 else L.F32
    o.loop_mode = _loop_mode(loop_mode)
    p_out = pressure_out if pressure_out is not None else torch.empty(N, dtype=torch.float64,
                                                                    device=dev)
    u_out = g_out = None
    if not light:
        u_out = torch.empty(N, dtype=torch.float64, device=dev)
        g_out = torch.empty(N, dtype=torch.float64, device=dev)
    hist = None
    hcap = 0
    if record_history:
        hcap = int(max_iter) + 1
        hist = np.zeros(hcap, dtype=np.float64)
    res = L.Result()
    L.check(L.lib().aspher_solve(
        op.handle, C.byref(o), _ptr(g0), C.c_double(float(p_nominal)), _ptr(p_init),
        _ptr(p_out), _ptr(u_out), _ptr(g_out),
        hist.ctypes.data_as(C.c_void_p) if hist is not None else C.c_void_p(0), hcap,
        C.byref(res), _stream()))
    h = hist[:res.history_len].copy() if hist is not None else None
    return ContactResult(res, op.Ns, p_out, u_out, g_out, h)


def _loop_mode(mode):
    if mode not in ("graph", "eager"):
        raise ValueError("loop_mode must be 'graph' or 'eager'")
    return 0 if mode == "graph" else 1


def _opts(tol, max_iter, use_pr, precond, keep_best, dtype, precond_radius=2, light=True,
          loop_mode="graph"):
    o = L.SolveOpts()
    L.lib().aspher_solve_opts_default(C.byref(o))
    o.tol = float(tol)
    o.max_iter = int(max_iter)
    o.use_pr = int(bool(use_pr))
    o.light = int(bool(light))
    o.keep_best = int(bool(keep_best))
    if precond not in L.PRECOND:
        raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
    o.precond = L.PRECOND[precond]
    o.precond_radius = int(precond_radius)
    o.dtype = L.F64 if dtype == torch.float64 else L.F32
    o.loop_mode = _loop_mode(loop_mode)
    return o


def solve_device_batch(op, g0s, p_nominals, tol=1e-8, max_iter=5000, use_pr=True,
                       precond="none", p_inits=None, dtype=torch.float64, keep_best=True,
                       pressures_out=None, loop_mode="graph"):
    """Batched solve_contact_impl<Real>: the problems g0s[b] (device fields
    of ``dtype``) with loads p_nominals[b] on one operator, solved together
    in one loop graph.  Returns one ContactResult per problem (pressure on
    the device; no displacement / gap fields)."""
    B = len(g0s)
    if B < 1 or len(p_nominals) != B:
        raise ValueError("solve_device_batch: need one p_nominal per gap")
    N = op.N
    g0s = [g.to(dtype).contiguous().reshape(-1) for g in g0s]
    for g in g0s:
        if g.numel() != N:
            raise ValueError("array has %d entries, expected %d" % (g.numel(), N))
    pis = None
    if p_inits is not None:
        pis = [None if p is None else p.to(dtype).contiguous().reshape(-1) for p in p_inits]
    outs = pressures_out or [torch.empty(N, dtype=torch.float64, device=g0s[0].device)
                             for _ in range(B)]
    o = _opts(tol, max_iter, use_pr, precond, keep_best, dtype, loop_mode=loop_mode)
    arr = C.c_void_p * B
    res = (L.Result * B)()
    L.check(L.lib().aspher_solve_batch(
        op.handle, C.byref(o), B, arr(*[g.data_ptr() for g in g0s]),
        (C.c_double * B)(*[float(p) for p in p_nominals]),
        arr(*[0 if p is None else p.data_ptr() for p in pis]) if pis else None,
        arr(*[p.data_ptr() for p in outs]), res, _stream()))
    return [ContactResult(res[b], op.Ns, outs[b]) for b in range(B)]


def solve_device_batch_mixed(op, g0s, p_nominals, tol=1e-6, float_tol=None, polish=True,
                             max_iter=5000, use_pr=True, precond="fourier", keep_best=True,
                             pressures_out=None, polish_tol=None, loop_mode="graph"):
    """Batched FP32 stage (FP64 reductions) + FP64 polish: the batched form
    of solve_device_mixed (same float_tol / polish_tol meaning).  g0s: FP64
    device fields.  Returns (final results, FP32-stage results)."""
    B = len(g0s)
    if B < 1 or len(p_nominals) != B:
        raise ValueError("solve_device_batch_mixed: need one p_nominal per gap")
    if polish_tol is not None and not (0.0 < polish_tol <= tol):
        raise ValueError("polish_tol must be in (0, tol]")
    N = op.N
    g0s = [g.to(torch.float64).contiguous().reshape(-1) for g in g0s]
    for g in g0s:
        if g.numel() != N:
            raise ValueError("array has %d entries, expected %d" % (g.numel(), N))
    outs = pressures_out or [torch.empty(N, dtype=torch.float64, device=g0s[0].device)
                             for _ in range(B)]
    o = _opts(tol if polish_tol is None or not polish else polish_tol, max_iter, use_pr,
              precond, keep_best, torch.float64, loop_mode=loop_mode)
    o.requested_tol = float(tol)
    arr = C.c_void_p * B
    res, resf = (L.Result * B)(), (L.Result * B)()
    L.check(L.lib().aspher_solve_batch_mixed(
        op.handle, C.byref(o), B, arr(*[g.data_ptr() for g in g0s]),
        (C.c_double * B)(*[float(p) for p in p_nominals]),
        C.c_double(float(tol if float_tol is None else float_tol)), int(bool(polish)),
        arr(*[p.data_ptr() for p in outs]), res, resf, _stream()))
    return ([ContactResult(res[b], op.Ns, outs[b]) for b in range(B)],
            [ContactResult(resf[b], op.Ns, None) for b in range(B)])


class ContactSolver:
    """``aspher.ContactSolver`` for backend='fft' / 'periodic' (bindings.cpp:805-834).

    The H-matrix / H2 / dense arguments are accepted for signature
    compatibility and ignored; any backend other than 'fft' or 'periodic'
    raises ValueError (those backends are not part of this build).
    """

    def __init__(self, grid_size, domain_size=1.0, E_star=1.0, eta=2.0, aca_tol=1e-6,
                 leaf_size=64, use_hmatrix=True, use_acagp=False, central_fraction=0.3,
                 inline_svd_tol=0.0, backend="", q=4, near_radius=1, h2_leaf_side=8):
        if grid_size <= 0:
            raise ValueError("grid_size must be positive")
        if not domain_size > 0.0:
            raise ValueError("domain_size must be positive")
        if not E_star > 0.0:
            raise ValueError("E_star must be positive")
        if backend == "":
            backend = "hmatrix" if use_hmatrix else "dense"
        if backend not in ("fft", "periodic"):
            raise ValueError("unknown backend: %s (aspher_b200 implements 'fft' and "
                             "'periodic')" % backend)
        self.Ns = int(grid_size)
        self.backend = backend
        self.op = Operator(backend, grid_size, domain_size, E_star)

    def matvec(self, p):
        """u = S p for a float64 array of shape (N,) or (Ns, Ns); returns (N,)."""
        v = _as_vector(p, self.Ns * self.Ns)
        dev = _dev()
        x = torch.from_numpy(v).to(dev)
        y = torch.empty_like(x)
        self.op.matvec_(x, y)
        return y.cpu().numpy()

    def solve(self, gap, p_nominal, tol=1e-8, max_iter=5000, use_pr=True, precond="none",
              p_init=None, *, precision="double", float_tol=None, polish_tol=None,
              reference_fp64=False):
        """Normal contact solve (bindings.cpp:186-234); always FP64 by default.

        ``precision`` (keyword-only extension): 'double' (reference),
        'float' (FP32 vectors and transforms, FP64 reductions) or
        'float_then_double' (FP32 to float_tol (default tol), then an FP64
        polish that certifies polish_tol (default tol); see
        solve_device_mixed).

        ``reference_fp64`` (keyword-only, for 'float' / 'float_then_double'):
        also run the plain FP64 solve of the same problem (same tol,
        preconditioner and warm start) and state the result's accuracy
        against it in ``pressure_rel_l2_vs_fp64`` (||p - p64|| / ||p64||),
        ``contact_area_error_vs_fp64`` (|A - A64|) and ``fp64_status``;
        without it those fields are None.
        """
        N = self.Ns * self.Ns
        if precond not in ("none", "", "fourier", "fourier-fft"):
            raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
        dev = _dev()
        g0d = _to_device_f64(gap, N, dev)
        p0 = None if p_init is None else _to_device_f64(p_init, N, dev)
        t0 = time.perf_counter()
        if precision == "double":
            r = solve_device(self.op, g0d, p_nominal, tol, max_iter, use_pr, precond, p0,
                             torch.float64)
        elif precision in ("float", "float_then_double"):
            r, _ = solve_device_mixed(self.op, g0d, p_nominal, tol, float_tol,
                                      precision == "float_then_double", max_iter, use_pr,
                                      precond, p0, polish_tol=polish_tol)
        else:
            raise ValueError("precision must be 'double', 'float' or 'float_then_double'")
        r.wall = time.perf_counter() - t0
        if reference_fp64 and precision != "double":
            rd = solve_device(self.op, g0d, p_nominal, tol, max_iter, use_pr, precond, p0,
                              torch.float64, light=True)
            pd = rd.pressure_device
            r.pressure_rel_l2_vs_fp64 = float(torch.linalg.norm(r.pressure_device - pd) /
                                              torch.linalg.norm(pd))
            r.contact_area_error_vs_fp64 = abs(r.contact_area - rd.contact_area)
            r.fp64_status = rd.status
        return r

    def block_layout(self):
        """(0, 6) float64 array: the reference returns block rows only for the
        'hmatrix' backend and an empty (0, 6) array for every other one
        (bindings.cpp:240-242)."""
        return np.zeros((0, 6), dtype=np.float64)

    def recompress(self, svd_tol):
        """No-op: the reference recompresses only 'hmatrix' operators
        (bindings.cpp:258-260)."""
        return None

    def hmatrix_info(self):
        inf = self.op.info()
        d = {"backend": self.backend, "n": int(inf.n)}
        if self.backend == "fft":
            d.update(padded_side=int(inf.padded_side), bytes=int(inf.bytes_total),
                     bytes_spectrum=int(inf.bytes_spectrum),
                     bytes_scratch=int(inf.bytes_scratch),
                     compression=float(inf.bytes_total) / (8.0 * inf.n * inf.n))
        else:
            d.update(periodic_x=True, periodic_y=True, bytes_scratch=int(inf.bytes_scratch))
        return d


def solve_device_mixed(op, g0, p_nominal, tol=1e-6, float_tol=None, polish=True,
                       max_iter=5000, use_pr=True, precond="fourier", p_init=None,
                       light=False, keep_best=None, g_ref=0.0, datum_mode="automatic",
                       datum=0.0, precond_radius=2, pressure_out=None, polish_tol=None,
                       loop_mode="graph"):
    """FP32 PK solve with FP64 reductions to ``float_tol`` (default: tol),
    then (polish) an FP64 PK solve warm-started from it that certifies
    ``polish_tol`` (default: tol; must be <= tol): the reference's
    float_then_double staging on one grid.  A polish_tol below tol buys
    pressure accuracy the certificate does not measure: FP32 rounding leaves
    a high-frequency pressure error (1e-5 .. 3e-5 relative at Ns=2048) that
    barely moves the Frank-Wolfe gap, and a few FP64 iterations past tol
    remove it.  ``requested_tol`` of the result stays tol.
    g0 / p_init: FP64 device tensors.  Returns (final, float_stage)."""
    N = op.N
    if g0.numel() != N:
        raise ValueError("array has %d entries, expected %d" % (g0.numel(), N))
    if precond not in L.PRECOND:
        raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
    dev = g0.device
    g0 = g0.to(torch.float64).contiguous().reshape(-1)
    if p_init is not None:
        p_init = p_init.to(device=dev, dtype=torch.float64).contiguous().reshape(-1)
        if p_init.numel() != N:
            raise ValueError("solve_contact: p_init size mismatch")
    if polish_tol is not None and not (0.0 < polish_tol <= tol):
        raise ValueError("polish_tol must be in (0, tol]")
    o = L.SolveOpts()
    L.lib().aspher_solve_opts_default(C.byref(o))
    o.tol = float(tol if polish_tol is None or not polish else polish_tol)
    o.requested_tol = float(tol)
    o.max_iter = int(max_iter)
    o.use_pr = int(bool(use_pr))
    o.light = int(bool(light))
    o.keep_best = int(not light) if keep_best is None else int(bool(keep_best))
    o.precond = L.PRECOND[precond]
    o.precond_radius = int(precond_radius)
    o.g_ref = float(g_ref)
    o.datum_mode = L.DATUM[datum_mode]
    o.datum = float(datum)
    o.loop_mode = _loop_mode(loop_mode)
    p_out = pressure_out if pressure_out is not None else torch.empty(N, dtype=torch.float64,
                                                                    device=dev)
    u_out = g_out = None
    if not light:
        u_out = torch.empty(N, dtype=torch.float64, device=dev)
        g_out = torch.empty(N, dtype=torch.float64, device=dev)
    res, resf = L.Result(), L.Result()
    ftol = float(tol if float_tol is None else float_tol)
    L.check(L.lib().aspher_solve_mixed(
        op.handle, C.byref(o), _ptr(g0), C.c_double(float(p_nominal)), _ptr(p_init),
        C.c_double(ftol), int(bool(polish)), _ptr(p_out), _ptr(u_out), _ptr(g_out),
        C.byref(res), C.byref(resf), _stream()))
    r = ContactResult(res, op.Ns, p_out, u_out, g_out)
    rf = ContactResult(resf, op.Ns, None)
    r.stage_stats = [dict(name="float", precision="float", iterations=rf.iterations,
                          matvec_count=rf.matvec_count, status=rf.status,
                          fw_error=rf.fw_error, penetration_error=rf.penetration_error)]
    if polish:
        r.stage_stats.append(dict(name="polish", precision="double",
                                  iterations=r.iterations - rf.iterations,
                                  status=r.status, fw_error=r.fw_error,
                                  penetration_error=r.penetration_error))
    return r, rf
