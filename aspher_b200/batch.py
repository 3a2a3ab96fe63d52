"""Many independent solves of uneven grid sizes and backends.

No reference counterpart (the reference solves one problem per call).
``solve_many`` is one call of the library's ``aspher_solve_many``, which
groups the problems by operator (backend, grid size); each group is one
batched solve on one operator (every kernel of the loop launched once for
the whole group, one CUDA-graph loop, per-instance convergence masks), and
the groups run concurrently, one host thread and one CUDA stream each
inside the library, so the small grids fill the SMs the large ones leave
idle.  Across GPUs the problems are dealt out by a greedy
longest-processing-time partition of their estimated cost (no collective:
each rank solves its own problems).
"""

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L
from .api import ContactResult, Operator, _stream
from .surfaces import self_affine_gap


def solve_cost(backend, Ns):
    """Relative cost estimate of one solve: Ns^2 log2(Ns) per apply (the
    free-space operator transforms a 2Ns grid: about twice the periodic)."""
    return (2.0 if backend == "fft" else 1.0) * Ns * Ns * math.log2(Ns)


def lpt_partition(costs, nbins):
    """Greedy LPT: indices sorted by decreasing cost, each to the bin with
    the smallest load so far (ties to the lowest bin).  Returns nbins lists
    of indices (each sorted)."""
    if nbins < 1:
        raise ValueError("nbins must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * nbins
    bins = [[] for _ in range(nbins)]
    for i in order:
        b = min(range(nbins), key=lambda k: (loads[k], k))
        bins[b].append(i)
        loads[b] += costs[i]
    return [sorted(b) for b in bins]


def uneven_problems(n=96, seed=2026, sizes=(256, 512, 1024, 2048),
                    weights=(0.4, 0.3, 0.2, 0.1), rms=0.002):
    """The uneven batch workload: Ns ~ categorical(sizes, weights),
    Hurst ~ U[0.6, 0.9], log p_nominal ~ U[ln 1e-3, ln 2e-2], backends
    alternating fft / periodic, surface seed 1000 + i (seeded synthetic
    self-affine gaps, |k| in [4, 64] cycles per domain)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        Ns = int(rng.choice(np.asarray(sizes), p=np.asarray(weights)))
        H = float(rng.uniform(0.6, 0.9))
        pn = float(math.exp(rng.uniform(math.log(1e-3), math.log(2e-2))))
        backend = "fft" if i % 2 == 0 else "periodic"
        out.append(dict(index=i, backend=backend, grid_size=Ns, hurst=H, p_nominal=pn,
                        seed=1000 + i, rms=rms))
    return out


def problem_gap(pr):
    return self_affine_gap(pr["grid_size"], hurst=pr["hurst"], rms=pr["rms"], seed=pr["seed"])


class Operators:
    """Per-process cache of operators keyed (backend, grid size) for one L, E*."""

    def __init__(self, domain_size=1.0, E_star=1.0):
        self.L = domain_size
        self.E = E_star
        self._ops = {}

    def get(self, backend, Ns):
        k = (backend, int(Ns))
        if k not in self._ops:
            self._ops[k] = Operator(backend, int(Ns), self.L, self.E)
        return self._ops[k]


def solve_many(problems, gaps, tol=1e-6, polish_tol=None, precond="fourier", max_iter=5000,
               precision="float_then_double", concurrent=True, operators=None,
               device=None, float_tol=None, domain_size=1.0, E_star=1.0):
    """Solve ``problems`` (dicts with backend, grid_size, p_nominal) with the
    matching ``gaps`` (device tensors or arrays of Ns^2 FP64 values) in one
    library call (``aspher_solve_many``): the library groups them per
    operator, solves each group as one batched solve and runs the groups
    concurrently on its own streams and host threads.  Returns the
    ContactResults in problem order (pressures on the device).  Work recorded
    on the caller's current stream afterwards runs after every group (so CUDA
    events on that stream bracket the whole batch).  ``operators`` is kept
    for signature compatibility: the library caches its operators itself."""
    del operators
    if len(problems) != len(gaps):
        raise ValueError("solve_many: one gap per problem")
    if precision not in L.MANY_PRECISION:
        raise ValueError("precision must be 'double', 'float' or 'float_then_double'")
    if precond not in L.PRECOND:
        raise ValueError("precond must be 'none', 'fourier' or 'fourier-fft'")
    n = len(problems)
    if n == 0:
        return []
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    arr = (L.Problem * n)()
    ins, outs = [], []
    for i, pr in enumerate(problems):
        if pr["backend"] not in L.BACKEND:
            raise ValueError("unknown backend: %s" % pr["backend"])
        Ns = int(pr["grid_size"])
        g = torch.as_tensor(gaps[i], dtype=torch.float64)
        # host gaps in pinned memory are copied asynchronously on the current
        # stream (the library's groups wait for it; the tensors stay
        # referenced until the synchronous call returns)
        g = g.to(dev, non_blocking=g.device.type == "cpu" and g.is_pinned())
        g = g.reshape(-1).contiguous()
        if g.numel() != Ns * Ns:
            raise ValueError("solve_many: problem %d: gap has %d entries, expected %d"
                             % (i, g.numel(), Ns * Ns))
        out = torch.empty(Ns * Ns, dtype=torch.float64, device=dev)
        ins.append(g)
        outs.append(out)
        arr[i] = L.Problem(L.BACKEND[pr["backend"]], Ns, float(pr.get("domain_size", domain_size)),
                           float(pr.get("E_star", E_star)), g.data_ptr(),
                           float(pr["p_nominal"]), out.data_ptr())
    o = L.ManyOpts()
    L.lib().aspher_many_opts_default(C.byref(o))
    o.precision = L.MANY_PRECISION[precision]
    o.tol = float(tol)
    o.float_tol = float(float_tol or 0.0)
    o.polish_tol = float(polish_tol or 0.0)
    o.max_iter = int(max_iter)
    o.precond = L.PRECOND[precond]
    o.concurrent = int(bool(concurrent))
    res, resf = (L.Result * n)(), (L.Result * n)()
    with torch.cuda.device(dev):
        L.check(L.lib().aspher_solve_many(n, arr, C.byref(o), res, resf, _stream()))
    out = []
    for i in range(n):
        Ns = int(problems[i]["grid_size"])
        r = ContactResult(res[i], Ns, outs[i])
        # the FP32 stage of a float_then_double solve (its iterations are
        # part of r.iterations)
        r.float_stage = (ContactResult(resf[i], Ns, None) if precision == "float_then_double"
                         else None)
        out.append(r)
    return out
