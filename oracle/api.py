"""``ContactSolver`` / ``solve_nested`` facade over the oracle.

Test infrastructure only (see ``oracle/__init__.py``).  Mirrors the pybind11
surface of ``python/bindings.cpp`` (class at :115-234, module defs at
:804-879) for the fft / periodic / dense backends, so the parity tests can
call the oracle and the CUDA product with the same arguments.
"""

import numpy as np

from .love import assemble_dense
from .nested import solve_contact_nested
from .operators import FFTOperator, PeriodicFFTOperator
from .precond import FourierPreconditioner, StencilPreconditioner
from .solver import SolveOptions, solve_contact_impl


class ContactSolver:
    def __init__(self, grid_size, domain_size=1.0, E_star=1.0, backend="fft",
                 **_unused):
        if grid_size <= 0:
            raise ValueError("grid_size must be positive")
        if not domain_size > 0.0:
            raise ValueError("domain_size must be positive")
        if not E_star > 0.0:
            raise ValueError("E_star must be positive")
        self.Ns = int(grid_size)
        self.backend = backend
        if backend == "fft":
            self.op = FFTOperator(grid_size, domain_size, E_star)
            self.mv = self.op.matvec
        elif backend == "periodic":
            self.op = PeriodicFFTOperator(grid_size, domain_size, E_star)
            self.mv = self.op.matvec
        elif backend == "dense":
            self.S = assemble_dense(grid_size, domain_size, E_star)
            self.mv = lambda x, dt=np.float64: (self.S @ np.asarray(x, np.float64)).astype(dt)
        else:
            raise ValueError("unknown backend: " + backend)

    def matvec(self, p):
        return self.mv(np.asarray(p, dtype=np.float64).reshape(-1))

    def solve(self, gap, p_nominal, tol=1e-8, max_iter=5000, use_pr=True,
              precond="none", p_init=None):
        N = self.Ns * self.Ns
        g0 = np.asarray(gap, dtype=np.float64).reshape(-1)
        if g0.size != N:
            raise ValueError(f"array has {g0.size} entries, expected {N}")
        pc = None
        if precond == "fourier":
            sp = StencilPreconditioner(self.Ns, 2)
            pc = lambda g, c: sp.apply(g, c, np.float64)
        elif precond == "fourier-fft":
            fp = FourierPreconditioner(self.Ns)
            pc = lambda g, c: fp.apply(g, c, np.float64)
        elif precond not in ("none", ""):
            raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
        opt = SolveOptions(tol=tol, max_iter=max_iter, use_pr=use_pr)
        p0 = None if p_init is None else np.asarray(p_init, np.float64).reshape(-1)
        r = solve_contact_impl(lambda x: self.mv(x, np.float64), g0, p_nominal,
                               opt, pc, p0, dtype=np.float64)
        r.pressure = r.pressure.reshape(self.Ns, self.Ns)
        return r


def solve_nested(grid_size, gap, p_nominal, domain_size=1.0, E_star=1.0,
                 coarsest=64, backend="fft", **kw):
    return solve_contact_nested(grid_size, domain_size, E_star, gap, p_nominal,
                                coarsest=coarsest, backend=backend, **kw)
