"""ctypes binding of libaspher_b200.so (the C ABI of include/aspher_b200.h).

The library is loaded from this package directory only; there is no CPU
fallback: if the shared object is missing or fails to load, every call into
the package raises.
"""

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaspher_b200.so")

ASPHER_OK = 0
ASPHER_EINVAL = -1
ASPHER_ECUDA = -2
ASPHER_EBUILD = -3
ASPHER_ETIMEOUT = -4

BACKEND = {"fft": 0, "periodic": 1}
F32, F64 = 0, 1
PRECOND = {"none": 0, "": 0, "stencil": 1, "fourier": 1, "fft": 2, "fourier-fft": 2}
DATUM = {"automatic": 0, "solver": 1, "caller": 2}
STATUS_NAMES = ("converged", "stagnated", "max_iterations", "nonpositive_curvature",
                "nonfinite", "verification_failed", "resource_limit")


class OpInfo(C.Structure):
    _fields_ = [("backend", C.c_int), ("grid_size", C.c_int), ("padded_side", C.c_int),
                ("n", C.c_int64), ("bytes_spectrum", C.c_int64),
                ("bytes_scratch", C.c_int64), ("bytes_total", C.c_int64),
                ("max_im_ratio", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("requested_tol", C.c_double), ("max_iter", C.c_int),
                ("use_pr", C.c_int), ("light", C.c_int), ("record_history", C.c_int),
                ("keep_best", C.c_int), ("load_tol", C.c_double), ("stall_limit", C.c_int),
                ("allow_tolerance_relaxation", C.c_int), ("precond", C.c_int),
                ("precond_radius", C.c_int), ("p_ref", C.c_double), ("g_ref", C.c_double),
                ("datum_mode", C.c_int), ("datum", C.c_double), ("dtype", C.c_int),
                ("loop_mode", C.c_int)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("status_reason", C.c_char * 32),
                ("iterations", C.c_int), ("converged", C.c_int),
                ("contact_fraction", C.c_double), ("mean_pressure", C.c_double),
                ("approach", C.c_double), ("objective", C.c_double), ("error", C.c_double),
                ("pk_error", C.c_double), ("fw_gap", C.c_double), ("fw_error", C.c_double),
                ("load_error", C.c_double), ("pressure_violation", C.c_double),
                ("penetration_error", C.c_double), ("requested_tol", C.c_double),
                ("effective_tol", C.c_double), ("p_ref", C.c_double), ("g_ref", C.c_double),
                ("matvec_count", C.c_int64), ("precond_count", C.c_int64),
                ("identification_steps", C.c_int), ("returned_best", C.c_int),
                ("history_len", C.c_int), ("time_total", C.c_double),
                ("mem_cg_state", C.c_int64), ("mem_best_iterate", C.c_int64),
                ("mem_contact_mask", C.c_int64), ("mem_output_arrays", C.c_int64),
                ("mem_peak", C.c_int64), ("time_build", C.c_double),
                ("time_coarse", C.c_double), ("active_rounds", C.c_int),
                ("active_fallback", C.c_int), ("time_candidate", C.c_double)]


class NestedOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int), ("use_pr", C.c_int),
                ("coarsest", C.c_int), ("q", C.c_int), ("leaf_side", C.c_int),
                ("precond", C.c_int), ("precond_engine", C.c_int),
                ("precond_radius", C.c_int), ("precond_occupancy_max", C.c_double),
                ("coarse_tol", C.c_double), ("single_precision", C.c_int),
                ("precision", C.c_int), ("float_floor", C.c_double),
                ("allow_tolerance_relaxation", C.c_int), ("light_result", C.c_int),
                ("record_error_history", C.c_int), ("active_set", C.c_int),
                ("active_delta", C.c_double), ("active_halo", C.c_int),
                ("active_max_rounds", C.c_int), ("active_all_levels", C.c_int),
                ("active_occupancy_max", C.c_double)]


class Stage(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("precision", C.c_char * 8), ("q", C.c_int),
                ("requested_tol", C.c_double), ("effective_tol", C.c_double),
                ("iterations", C.c_int), ("matvec_count", C.c_int64), ("seconds", C.c_double),
                ("status", C.c_int), ("fw_error", C.c_double),
                ("penetration_error", C.c_double), ("precond_dropped", C.c_int)]


class AdjointInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("contact_count", C.c_int),
                ("reserved", C.c_int), ("residual", C.c_double), ("mu", C.c_double),
                ("time", C.c_double)]


class Problem(C.Structure):
    _fields_ = [("backend", C.c_int), ("grid_size", C.c_int), ("domain_size", C.c_double),
                ("E_star", C.c_double), ("g0_dev", C.c_void_p), ("p_bar", C.c_double),
                ("pressure_dev", C.c_void_p)]


class ManyOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("tol", C.c_double), ("float_tol", C.c_double),
                ("polish_tol", C.c_double), ("max_iter", C.c_int), ("precond", C.c_int),
                ("precond_radius", C.c_int), ("concurrent", C.c_int)]


MANY_PRECISION = {"double": 0, "float": 1, "float_then_double": 2}


class TanResult(C.Structure):
    _fields_ = [("status", C.c_int), ("status_reason", C.c_char * 48), ("iterations", C.c_int),
                ("converged", C.c_int), ("error", C.c_double), ("delta_t", C.c_double * 2),
                ("q_mean", C.c_double * 2), ("n_stick", C.c_int), ("n_slip", C.c_int),
                ("n_open", C.c_int), ("cone_violation", C.c_double),
                ("stick_residual", C.c_double), ("slip_residual", C.c_double),
                ("proj_residual", C.c_double), ("force_error", C.c_double), ("rho", C.c_double),
                ("s_ref", C.c_double), ("w_ref", C.c_double), ("kkt_tol", C.c_double)]


# exported symbol -> (restype, argtypes)
SIGNATURES = {
    "aspher_abi_version": (C.c_int, []),
    "aspher_last_error": (C.c_char_p, []),
    "aspher_launch_count": (C.c_int64, []),
    "aspher_status_string": (C.c_char_p, [C.c_int]),
    "aspher_op_create": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double,
                                   C.POINTER(C.c_void_p)]),
    "aspher_op_create_ex": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                      C.POINTER(C.c_void_p)]),
    "aspher_op_destroy": (C.c_int, [C.c_void_p]),
    "aspher_op_matvec": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "aspher_op_get_info": (C.c_int, [C.c_void_p, C.POINTER(OpInfo)]),
    "aspher_op_love_table": (C.c_int, [C.c_void_p, C.c_void_p]),
    "aspher_op_set_variants": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "aspher_op_get_variants": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "aspher_op_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "aspher_precond_apply": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    "aspher_stencil_taps": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int,
                                      C.POINTER(C.c_int)]),
    "aspher_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
    "aspher_solve": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.c_double,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_int, C.POINTER(Result), C.c_void_p]),
    "aspher_solve_mixed": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.c_double,
                                     C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.POINTER(Result), C.POINTER(Result),
                                     C.c_void_p]),
    "aspher_solve_batch": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_int,
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_double),
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                     C.POINTER(Result), C.c_void_p]),
    "aspher_solve_batch_mixed": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_int,
                                           C.POINTER(C.c_void_p), C.POINTER(C.c_double),
                                           C.c_double, C.c_int, C.POINTER(C.c_void_p),
                                           C.POINTER(Result), C.POINTER(Result), C.c_void_p]),
    "aspher_tan_create": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.POINTER(C.c_void_p)]),
    "aspher_tan_destroy": (C.c_int, [C.c_void_p]),
    "aspher_tan_matvec": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "aspher_tan_max_im_ratio": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "aspher_solve_tangential": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                          C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                          C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.POINTER(TanResult), C.c_void_p]),
    "aspher_tan_tables": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "aspher_many_opts_default": (None, [C.POINTER(ManyOpts)]),
    "aspher_solve_many": (C.c_int, [C.c_int, C.POINTER(Problem), C.POINTER(ManyOpts),
                                    C.POINTER(Result), C.POINTER(Result), C.c_void_p]),
    "aspher_adjoint": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                 C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double),
                                 C.POINTER(AdjointInfo), C.c_void_p]),
    "aspher_periodic_matvec_noalloc": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_int,
                                                 C.c_void_p, C.c_void_p, C.c_void_p]),
    "aspher_nested_opts_default": (None, [C.POINTER(NestedOpts)]),
    "aspher_solve_nested": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                      C.c_double, C.POINTER(NestedOpts), C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.POINTER(Result), C.POINTER(Stage), C.c_int,
                                      C.POINTER(C.c_int), C.c_void_p]),
    "aspher_stencil_for_level": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double]),
    "aspher_operator_cache_clear": (C.c_int, []),
}

_lib = None


class AspherError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    """The loaded library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "libaspher_b200.so not found at %s; build it with "
                "`python -m aspher_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (rt, at) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = rt
            f.argtypes = at
        _lib = L
    return _lib


def check(code):
    if code != ASPHER_OK:
        msg = lib().aspher_last_error().decode(errors="replace")
        if code == ASPHER_EINVAL:
            raise ValueError(msg)
        raise AspherError(code, msg)
