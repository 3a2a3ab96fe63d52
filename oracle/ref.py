"""The reference's own C++ hot path, loaded from ``oracle/_ref`` -- TEST
INFRASTRUCTURE ONLY.

``oracle/Makefile`` compiles the unmodified reference sources
(``src/contact_solver.cpp``, ``src/fft_operator.cpp``,
``src/periodic_fft_operator.cpp``, ``src/boussinesq_kernel.cpp``,
``src/stencil_precond.cpp``, ``src/fourier_precond.cpp``,
``src/cerruti_kernel.cpp``, ``src/friction_solve.cpp``, with the vendored
pocketfft and OpenMP) against the project's Eigen-API shim
(``oracle/eigen_shim``) and the C-ABI harness ``oracle/ref_harness.cpp`` into
``oracle/_ref/libaspher_ref.so``.  ``ContactSolver`` below mirrors the
reference's pybind11 class (``python/bindings.cpp:115-214``) for the fft and
periodic backends.  Only tests, ``smoke()`` and bench.py's reference and
CPU-baseline legs use it, as the checker and the timed CPU baseline.

``available()`` is False where the library was not built (the reference tree
is needed to build it); callers then fall back to the numpy restatement in
this package.
"""

import ctypes
import os

import numpy as np

from .solver import ContactResult

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libaspher_ref.so")
STATUS = ("converged", "stagnated", "max_iterations", "nonpositive_curvature", "nonfinite",
          "verification_failed", "resource_limit")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.c_void_p


def build(ref_root="/root/reference"):
    """Compile the library (make -C oracle) when the reference tree exists."""
    import subprocess
    if not os.path.isdir(os.path.join(ref_root, "src")):
        return False
    p = subprocess.run(["make", "-s", "-C", HERE, "REF=" + ref_root], capture_output=True,
                       text=True)
    if p.returncode != 0:
        raise RuntimeError("reference build failed:\n" + p.stderr[-4000:])
    return True


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libaspher_ref.so is not built (make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        L.aref_op_create.restype = ctypes.c_void_p
        L.aref_op_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double]
        L.aref_op_destroy.argtypes = [ctypes.c_void_p]
        L.aref_op_matvec.argtypes = [ctypes.c_void_p, ctypes.c_int, _F, _F]
        L.aref_love_table.argtypes = [ctypes.c_void_p, _D]
        L.aref_precond_apply.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D,
                                         ctypes.c_void_p, _D]
        L.aref_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_double, _D,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D,
                                 _D, ctypes.c_int, ctypes.c_char_p]
        L.aref_last_error.restype = ctypes.c_char_p
        L.aref_status_string.restype = ctypes.c_char_p
        L.aref_project_simplex.restype = ctypes.c_double
        L.aref_project_simplex.argtypes = [_D, ctypes.c_int64, ctypes.c_double]
        L.aref_set_threads.argtypes = [ctypes.c_int]
        L.aref_cerruti_tables.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, _D, _D, _D]
        L.aref_tan_create.restype = ctypes.c_void_p
        L.aref_tan_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double]
        L.aref_tan_destroy.argtypes = [ctypes.c_void_p]
        L.aref_tan_matvec.argtypes = [ctypes.c_void_p, _D, _D]
        L.aref_solve_tangential.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                            _D, _D, ctypes.c_char_p]
        for f in (L.aref_cerruti_uxx, L.aref_cerruti_uxy):
            f.restype = ctypes.c_double
        L.aref_cerruti_uxx.argtypes = [ctypes.c_double] * 5
        L.aref_cerruti_uxy.argtypes = [ctypes.c_double] * 4
        _lib = L
    return _lib


def threads():
    return int(lib().aref_max_threads())


def set_threads(n):
    lib().aref_set_threads(int(n))


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def project_load_simplex(y, P_total):
    """project_load_simplex<double> (src/contact_solver.cpp:31-60); returns
    (projected copy, threshold)."""
    y = np.ascontiguousarray(y, np.float64).copy()
    th = lib().aref_project_simplex(_dp(y), y.size, float(P_total))
    return y, th


def cerruti_tables(Ns, L=1.0, E_star=1.0, nu=0.3):
    """CerrutiKernel's signed offset tables (xx, yy, xy), each indexed
    [dy + Ns - 1, dx + Ns - 1] for offsets in (-Ns, Ns)."""
    W = 2 * Ns - 1
    xx, yy, xy = (np.empty(W * W) for _ in range(3))
    if lib().aref_cerruti_tables(int(Ns), float(L), float(E_star), float(nu), _dp(xx), _dp(yy),
                                 _dp(xy)) != 0:
        raise ValueError(lib().aref_last_error().decode())
    return xx.reshape(W, W), yy.reshape(W, W), xy.reshape(W, W)


def cerruti_uxx(x, y, a, b, nu):
    return lib().aref_cerruti_uxx(float(x), float(y), float(a), float(b), float(nu))


def cerruti_uxy(x, y, a, b):
    return lib().aref_cerruti_uxy(float(x), float(y), float(a), float(b))


_TAN_FIELDS = ("status", "iterations", "converged", "error", "delta_x", "delta_y", "qmean_x",
               "qmean_y", "n_stick", "n_slip", "n_open", "cone_violation", "stick_residual",
               "slip_residual", "proj_residual", "force_error", "rho", "s_ref", "w_ref",
               "kkt_tol")


class Tangential:
    """The tangential (Cerruti) FFT operator of src/tangential_operator.cpp,
    restated in the harness on the reference's FFT engine and CerrutiKernel,
    with the reference's solve_tangential (src/friction_solve.cpp) on it."""

    def __init__(self, grid_size, domain_size=1.0, E_star=1.0, nu=0.3):
        self.Ns = int(grid_size)
        self._h = lib().aref_tan_create(self.Ns, float(domain_size), float(E_star), float(nu))
        if not self._h:
            raise ValueError(lib().aref_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().aref_tan_destroy(self._h)
            self._h = None

    def matvec(self, q):
        q = np.ascontiguousarray(np.asarray(q, np.float64).reshape(-1))
        u = np.empty_like(q)
        lib().aref_tan_matvec(self._h, _dp(q), _dp(u))
        return u

    def solve(self, s, force_control, target, tol=1e-8, max_iter=5000, use_pr=True,
              kkt_tol=0.0, q_init=None):
        """solve_tangential(C, s, force_control, target, tol, max_iter, use_pr,
        {}, q_init) unpreconditioned; returns (q (2N,), dict of the result
        fields)."""
        s = np.ascontiguousarray(np.asarray(s, np.float64).reshape(-1))
        q = np.empty(2 * s.size, np.float64)
        qi = None if q_init is None else np.ascontiguousarray(
            np.asarray(q_init, np.float64).reshape(-1))
        if qi is not None and qi.size != 2 * s.size:
            raise ValueError("q_init has %d entries, expected %d" % (qi.size, 2 * s.size))
        out = np.zeros(len(_TAN_FIELDS), np.float64)
        reason = ctypes.create_string_buffer(64)
        rc = lib().aref_solve_tangential(self._h, _dp(s), int(bool(force_control)),
                                         float(target[0]), float(target[1]), float(tol),
                                         int(max_iter), int(bool(use_pr)), float(kkt_tol),
                                         None if qi is None else qi.ctypes.data, _dp(q), _dp(out),
                                         reason)
        if rc != 0:
            raise ValueError(lib().aref_last_error().decode())
        d = dict(zip(_TAN_FIELDS, out.tolist()))
        d["status"] = STATUS[int(d["status"])]
        d["status_reason"] = reason.value.decode()
        for k in ("iterations", "n_stick", "n_slip", "n_open"):
            d[k] = int(d[k])
        d["converged"] = bool(d["converged"])
        return q, d


_SCALARS = ("status", "iterations", "converged", "contact_fraction", "mean_pressure",
            "approach", "objective", "error", "fw_gap", "fw_error", "load_error",
            "pressure_violation", "penetration_error", "requested_tol", "effective_tol",
            "p_ref", "g_ref", "matvec_count", "precond_count", "identification_steps",
            "returned_best", "time_total", "history_len")


class ContactSolver:
    """ContactSolver(grid_size, domain_size, E_star, backend) for backend
    "fft" / "periodic" on the reference's own C++ (python/bindings.cpp:119-148)."""

    def __init__(self, grid_size, domain_size=1.0, E_star=1.0, backend="fft", **_unused):
        if backend not in ("fft", "periodic"):
            raise ValueError("unknown backend: " + backend)
        self.Ns = int(grid_size)
        self.backend = backend
        self._h = lib().aref_op_create(0 if backend == "fft" else 1, self.Ns, float(domain_size),
                                       float(E_star))
        if not self._h:
            raise ValueError(lib().aref_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().aref_op_destroy(self._h)
            self._h = None

    def matvec(self, p, dtype=np.float64):
        x = np.ascontiguousarray(np.asarray(p).reshape(-1), dtype=dtype)
        y = np.empty_like(x)
        rc = lib().aref_op_matvec(self._h, 1 if dtype == np.float64 else 0, x.ctypes.data,
                                  y.ctypes.data)
        if rc != 0:
            raise RuntimeError(lib().aref_last_error().decode())
        return y

    def love_table(self):
        t = np.empty(self.Ns * self.Ns, np.float64)
        if lib().aref_love_table(self._h, _dp(t)) != 0:
            raise ValueError(lib().aref_last_error().decode())
        return t.reshape(self.Ns, self.Ns)

    def precond_apply(self, g, contact, precond="fourier", radius=2):
        g = np.ascontiguousarray(np.asarray(g).reshape(-1), np.float64)
        c = np.ascontiguousarray(np.asarray(contact).reshape(-1) != 0, np.uint8)
        z = np.empty_like(g)
        rc = lib().aref_precond_apply(self._h, 1 if precond == "fourier" else 2, int(radius),
                                      _dp(g), c.ctypes.data, _dp(z))
        if rc != 0:
            raise ValueError(lib().aref_last_error().decode())
        return z

    def solve(self, gap, p_nominal, tol=1e-8, max_iter=5000, use_pr=True, precond="none",
              p_init=None, dtype=np.float64, light=False, record_history=False,
              keep_best=True, radius=2, stall_limit=200, g_ref=0.0, p_ref=0.0, load_tol=0.0):
        """ContactSolver.solve (python/bindings.cpp:180-228): solve_contact with
        default SolveOptions; dtype=np.float32 runs solve_contact_impl<float>.
        The keyword options set the SolveOptions fields of the same names."""
        N = self.Ns * self.Ns
        g0 = np.ascontiguousarray(np.asarray(gap, dtype=np.float64).reshape(-1))
        if g0.size != N:
            raise ValueError(f"array has {g0.size} entries, expected {N}")
        pc = {"none": 0, "": 0, "fourier": 1, "fourier-fft": 2}.get(precond)
        if pc is None:
            raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
        p0 = None if p_init is None else np.ascontiguousarray(
            np.asarray(p_init, np.float64).reshape(-1))
        p = np.empty(N, np.float64)
        disp = None if light else np.empty(N, np.float64)
        gapo = None if light else np.empty(N, np.float64)
        out = np.zeros(len(_SCALARS) + 1, np.float64)
        cap = max_iter + 2 if record_history else 0
        hist = np.zeros(max(cap, 1), np.float64)
        reason = ctypes.create_string_buffer(64)
        opt = np.array([tol, max_iter, bool(use_pr), bool(light), bool(record_history),
                        bool(keep_best), stall_limit, g_ref, p_ref, load_tol], np.float64)
        rc = lib().aref_solve(self._h, 1 if dtype == np.float64 else 0, _dp(g0), float(p_nominal),
                              _dp(opt), opt.size, pc, int(radius), _dp(p0), _dp(p), _dp(disp),
                              _dp(gapo), _dp(out), _dp(hist), cap, reason)
        if rc != 0:
            raise ValueError(lib().aref_last_error().decode())
        v = dict(zip(_SCALARS, out.tolist()))
        r = ContactResult()
        r.pressure = p.reshape(self.Ns, self.Ns)
        r.displacement = disp
        r.gap = gapo
        r.status = STATUS[int(v["status"])]
        r.status_reason = reason.value.decode()
        r.iterations = int(v["iterations"])
        r.converged = bool(v["converged"])
        for k in ("contact_fraction", "mean_pressure", "approach", "objective", "error",
                  "fw_gap", "fw_error", "load_error", "pressure_violation", "penetration_error",
                  "requested_tol", "effective_tol", "p_ref", "g_ref", "time_total"):
            setattr(r, k, float(v[k]))
        r.pk_error = r.error
        r.matvec_count = int(v["matvec_count"])
        r.precond_count = int(v["precond_count"])
        r.identification_steps = int(v["identification_steps"])
        r.returned_best = bool(v["returned_best"])
        r.error_history = hist[:int(v["history_len"])].tolist() if record_history else []
        return r
