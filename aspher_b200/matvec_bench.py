"""Operator-apply timing (and a small, self-contained workload for ncu).

    python -m aspher_b200.matvec_bench --backend fft --ns 4096 --dtype f32 --iters 20

Times ``iters`` applies y = S x with CUDA events on the launching stream,
writing a 256 MB buffer between applies so every apply starts with a cold
L2, and prints one JSON line: mean / min apply time and the algorithmic
bandwidth of the row-column model (free space 12 b N bytes per apply,
periodic 6 b N; b = bytes per real).
"""

import argparse
import json
import statistics

import torch

from .api import Operator


def run(backend, ns, dtype, iters, warmup=3, flush=True, variants=None, op=None):
    dt = torch.float32 if dtype == "f32" else torch.float64
    b = 4 if dtype == "f32" else 8
    op = op if op is not None else Operator(backend, ns)
    if variants is not None:
        op.set_variants(variants[0], variants[1], dt)
    N = ns * ns
    xs = [torch.randn(N, dtype=dt, device="cuda") for _ in range(2)]
    y = torch.empty(N, dtype=dt, device="cuda")
    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for i in range(warmup):
        op.matvec_(xs[i % 2], y)
    torch.cuda.synchronize()
    ts = []
    for i in range(iters):
        if flush:
            buf.zero_()
        a = torch.cuda.Event(enable_timing=True)
        c = torch.cuda.Event(enable_timing=True)
        a.record()
        op.matvec_(xs[i % 2], y)
        c.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(c) / 1e3)
    model = (12 if backend == "fft" else 6) * b * N
    t = statistics.mean(ts)
    rv, cv, ct = op.variants(dt)
    return dict(backend=backend, ns=ns, dtype=dtype, iters=iters, variants=[rv, cv, ct],
                ms_mean=t * 1e3,
                ms_min=min(ts) * 1e3, alg_bytes=model, gbs=model / t / 1e9,
                gbs_best=model / min(ts) / 1e9)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--backend", default="fft", choices=("fft", "periodic"))
    ap.add_argument("--ns", type=int, default=2048)
    ap.add_argument("--dtype", default="f32", choices=("f32", "f64"))
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--sweep", action="store_true",
                    help="all backends x dtypes x Ns in {512..8192}")
    ap.add_argument("--variants", action="store_true",
                    help="with --sweep: time every (row, column) launch-variant pair")
    a = ap.parse_args()
    if a.sweep and a.variants:
        for backend in ("fft", "periodic"):
            for dtype in ("f32", "f64"):
                for ns in (256, 512, 1024, 2048, 4096, 8192):
                    op = Operator(backend, ns)
                    best = None
                    for cv in range(4):
                        for rv in range(4):
                            r = run(backend, ns, dtype, a.iters, a.warmup, variants=(rv, cv),
                                    op=op)
                            print(json.dumps(r), flush=True)
                            if best is None or r["ms_mean"] < best["ms_mean"]:
                                best = r
                    print(json.dumps(dict(best=best)), flush=True)
                    del op
        return
    if a.sweep:
        for backend in ("fft", "periodic"):
            for dtype in ("f32", "f64"):
                for ns in (512, 1024, 2048, 4096, 8192):
                    print(json.dumps(run(backend, ns, dtype, a.iters, a.warmup)), flush=True)
    else:
        print(json.dumps(run(a.backend, a.ns, a.dtype, a.iters, a.warmup)), flush=True)


if __name__ == "__main__":
    main()
