"""Many independent solves of uneven grid sizes and backends.

No reference counterpart (the reference solves one problem per call).  The
problems are grouped by (backend, grid size); each group is one batched
solve on one operator (``aspher_solve_batch_mixed``: every kernel of the
loop launched once for the whole group, one CUDA-graph loop, per-instance
convergence masks), and the groups run concurrently, one host thread and
one CUDA stream each, so the small grids fill the SMs the large ones leave
idle.  Across GPUs the problems are dealt out by a greedy
longest-processing-time partition of their estimated cost (no collective:
each rank solves its own problems).
"""

import concurrent.futures as cf
import math

import numpy as np
import torch

from .api import Operator, solve_device_batch, solve_device_batch_mixed
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
               device=None, float_tol=None):
    """Solve ``problems`` (dicts with backend, grid_size, p_nominal) with the
    matching ``gaps`` (device tensors or arrays of Ns^2 FP64 values).
    Returns the ContactResults in problem order (pressures on the device).
    Work recorded on the caller's current stream afterwards runs after every
    group (so CUDA events on that stream bracket the whole batch)."""
    if len(problems) != len(gaps):
        raise ValueError("solve_many: one gap per problem")
    if precision not in ("double", "float", "float_then_double"):
        raise ValueError("precision must be 'double', 'float' or 'float_then_double'")
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    ops = operators or Operators()
    groups = {}
    for i, pr in enumerate(problems):
        groups.setdefault((pr["backend"], int(pr["grid_size"])), []).append(i)
    # Everything that allocates or copies is done here, before any worker
    # starts: the operators, the groups' streams, gaps and outputs.  The
    # workers then only run the library's batched solves (which serialise
    # their own graph captures and set-up against each other).
    caller = torch.cuda.current_stream(dev)
    streams, inputs, outputs = {}, {}, {}
    for key, idx in groups.items():
        ops.get(*key)
        streams[key] = torch.cuda.Stream(device=dev)
        inputs[key] = [torch.as_tensor(gaps[i], dtype=torch.float64).to(dev).reshape(-1)
                       for i in idx]
        N = key[1] * key[1]
        outputs[key] = [torch.empty(N, dtype=torch.float64, device=dev) for _ in idx]
    torch.cuda.synchronize(dev)
    results = [None] * len(problems)
    done = []

    def run_group(key):
        b, Ns = key
        idx = groups[key]
        op = ops.get(b, Ns)
        stream = streams[key]
        stream.wait_stream(caller)
        with torch.cuda.device(dev), torch.cuda.stream(stream):
            g = inputs[key]
            pn = [problems[i]["p_nominal"] for i in idx]
            if precision == "double":
                rs = solve_device_batch(op, g, pn, tol=tol, max_iter=max_iter, precond=precond,
                                        dtype=torch.float64, keep_best=False,
                                        pressures_out=outputs[key])
            else:
                rs, _ = solve_device_batch_mixed(op, g, pn, tol=tol, float_tol=float_tol,
                                                 max_iter=max_iter,
                                                 precond=precond, keep_best=False,
                                                 polish=precision == "float_then_double",
                                                 polish_tol=polish_tol,
                                                 pressures_out=outputs[key])
            ev = torch.cuda.Event()
            ev.record(stream)
            done.append(ev)
        for i, r in zip(idx, rs):
            results[i] = r

    keys = sorted(groups, key=lambda k: -len(groups[k]) * solve_cost(k[0], k[1]))
    if concurrent and len(keys) > 1:
        with cf.ThreadPoolExecutor(len(keys)) as ex:
            for f in [ex.submit(run_group, k) for k in keys]:
                f.result()
    else:
        for k in keys:
            run_group(k)
    for ev in done:
        caller.wait_event(ev)
    return results
