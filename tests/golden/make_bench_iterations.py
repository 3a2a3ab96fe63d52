"""Oracle (FP64) iteration counts of the Ns=2048 benchmark problems.

bench.py's reference arm and CPU baseline time a bounded sample of oracle
PCG iterations (a full Ns=2048 oracle solve takes minutes) and scale it to a
whole solve with these counts.  Problems: backend in {fft, periodic},
p_nominal in {0.001, 0.005, 0.02}, self-affine surface seed 42 (H=0.8,
rms 0.002, |k| in [4, 64] cycles/domain), tol 1e-6, precond "fourier"
(13-tap stencil), FP64.  Run: python tests/golden/make_bench_iterations.py
"""

import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from aspher_b200.surfaces import self_affine_gap  # noqa: E402  (numpy only)
from oracle.api import ContactSolver  # noqa: E402

NS, TOL = 2048, 1e-6
LOADS = (0.001, 0.005, 0.02)


def main():
    out = {}
    g0 = self_affine_gap(NS, hurst=0.8, rms=0.002, seed=42)
    for backend in ("fft", "periodic"):
        s = ContactSolver(NS, backend=backend)
        for pbar in LOADS:
            t0 = time.perf_counter()
            r = s.solve(g0, pbar, tol=TOL, precond="fourier")
            dt = time.perf_counter() - t0
            key = "%s_%g" % (backend, pbar)
            out[key] = dict(iterations=r.iterations, matvec_count=r.matvec_count,
                            status=r.status, contact_area=r.contact_area,
                            seconds=round(dt, 2))
            print(key, out[key], flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bench_iterations.json")
    with open(path, "w") as f:
        json.dump(dict(ns=NS, tol=TOL, precond="fourier", seed=42, problems=out), f, indent=1)
    print(path)


if __name__ == "__main__":
    main()
