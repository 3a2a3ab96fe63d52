"""Golden fixtures of the Ns=2048 single-solve problems, made by the
reference's own C++ (oracle/_ref/libaspher_ref.so; build it with
``make -C oracle``).

Problems: backend in {fft, periodic} x p_nominal in {0.001, 0.005, 0.02} on
the seeded self-affine surface (seed 42, H=0.8, rms 0.002, |k| in [4, 64]
cycles/domain, L = E* = 1), precond "fourier" (13-tap stencil), FP64, the
reference's ContactSolver.solve: once at tol 1e-6 (the benchmark tolerance)
and once at tol 1e-10 (a tight solution to measure pressure errors against).

Written to ``tests/golden/ref_ns2048.npz`` (compressed) and
``tests/golden/ref_ns2048.json``:
  * per problem (json): iterations, status, contact area, certificates,
    sum and 2-norm of the pressure of both solves, the tol 1e-6 solve's
    rel-L2 distance to the tight one (full grid, on the sample, on blocks);
  * per problem (npz): ``<key>_idx``: 16384 cells drawn (seeded) from the
    union of both solves' contact sets; ``<key>_p6`` / ``<key>_p10``: the two
    pressures there (float64); ``<key>_blk``: the tight pressure averaged
    over 16x16 blocks (128 x 128, float32).
Run: python tests/golden/make_ref_fixtures.py   (about 10 min on 8 cores)
"""

import json
import os
import sys
import time
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from aspher_b200.surfaces import self_affine_gap  # noqa: E402  (numpy only)
from oracle import ref  # noqa: E402

NS = 2048
LOADS = (0.001, 0.005, 0.02)
NSAMPLE = 16384
BLK = 16


def block_avg(p, b=BLK):
    n = p.shape[0] // b
    return p.reshape(n, b, n, b).mean(axis=(1, 3))


def sample_idx(key, p6, p10):
    cand = np.flatnonzero((p6.reshape(-1) > 0) | (p10.reshape(-1) > 0))
    rng = np.random.default_rng(zlib.crc32(key.encode()))
    k = min(NSAMPLE, cand.size)
    return np.sort(rng.choice(cand, size=k, replace=False)).astype(np.int32)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main():
    g0 = self_affine_gap(NS, hurst=0.8, rms=0.002, seed=42)
    meta = {"ns": NS, "seed": 42, "precond": "fourier", "threads": ref.threads(),
            "generator": "reference C++ (oracle/_ref) via oracle/ref.py", "problems": {}}
    arrays = {}
    for backend in ("fft", "periodic"):
        s = ref.ContactSolver(NS, backend=backend)
        for pbar in LOADS:
            key = "%s_%g" % (backend, pbar)
            t0 = time.perf_counter()
            r6 = s.solve(g0, pbar, tol=1e-6, precond="fourier", light=True)
            t6 = time.perf_counter() - t0
            t0 = time.perf_counter()
            r10 = s.solve(g0, pbar, tol=1e-10, max_iter=20000, precond="fourier", light=True)
            t10 = time.perf_counter() - t0
            p6, p10 = r6.pressure, r10.pressure
            idx = sample_idx(key, p6, p10)
            b10 = block_avg(p10)
            rec = {}
            for tag, r, p, t in (("tol6", r6, p6, t6), ("tol10", r10, p10, t10)):
                rec[tag] = dict(iterations=r.iterations, status=r.status,
                                contact_area=r.contact_area, fw_error=r.fw_error,
                                penetration_error=r.penetration_error,
                                load_error=r.load_error, sum_p=float(p.sum()),
                                norm_p=float(np.linalg.norm(p)), seconds=round(t, 2))
            rec["tol6_vs_tol10"] = dict(full=rel(p6, p10),
                                        sample=rel(p6.reshape(-1)[idx], p10.reshape(-1)[idx]),
                                        blocks=rel(block_avg(p6), b10))
            meta["problems"][key] = rec
            arrays[key + "_idx"] = idx
            arrays[key + "_p6"] = p6.reshape(-1)[idx]
            arrays[key + "_p10"] = p10.reshape(-1)[idx]
            arrays[key + "_blk"] = b10.astype(np.float32)
            print(key, json.dumps(rec), flush=True)
    np.savez_compressed(os.path.join(HERE, "ref_ns2048.npz"), **arrays)
    with open(os.path.join(HERE, "ref_ns2048.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
