"""Benchmark: certified contact solves per second on B200 (one JSON line).

Workload (per GPU): the Ns=2048 single-solve configuration -- free-space
``fft`` and ``periodic`` backends x p_nominal in {0.001, 0.005, 0.02} on a
seeded self-affine surface (H=0.8, rms 0.002, |k| in [4, 64] cycles/domain,
L = E* = 1), tol 1e-6, 13-tap stencil preconditioner.  One step solves those
6 problems with the product path: FP32 operator / CG with FP64-accumulated
reductions, then an FP64 polish that certifies tol on the FP64 operator.
``value`` = certified solves/s with the gaps resident in HBM; ``e2e`` = the
same through ``ContactSolver.solve`` with the gap copied from pinned host
memory and the pressure read back every solve.  The plain FP64 GPU solve
of the same problems is timed as the comparator.  Ranks solve disjoint
problem sets (seed 42 + 1000*rank): weak scaling, no collective on the
data path.

``--impl reference`` times the reference algorithm's CPU implementation of
the same workload (the oracle restatement, all host cores for its FFTs):
each step runs a bounded sample of PCG iterations of one problem and scales
it by that problem's oracle iteration count (tests/golden/bench_iterations.json).
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("certified solves/s @Ns=2048 tol1e-6, FP32/batched vs FP64 GPU; "
          "matvec HBM GB/s")
NS = 2048
TOL = 1e-6
LOADS = (0.001, 0.005, 0.02)
BACKENDS = ("fft", "periodic")
SEED = 42


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--ns", type=int, default=NS)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---- clocks sampled during the timed region --------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
         "pci.bus_id")

    def __init__(self, bus_id=None):
        self.rows = []
        self.proc = None
        self.bus_id = bus_id

    def start(self):
        cmd = ["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
               "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = []
        mx = 0.0
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        rows = self.rows
        if self.bus_id:
            mine = [r for r in rows if len(r) > 9 and r[9].upper().endswith(self.bus_id[-7:])]
            if mine:
                rows = mine
            elif rows:
                first = rows[0][0]
                rows = [r for r in rows if r[0] == first]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def problem_gaps(Ns, rank):
    from aspher_b200.surfaces import self_affine_gap
    g = self_affine_gap(Ns, hurst=0.8, rms=0.002, k_lo=4.0, k_hi=64.0, seed=SEED + 1000 * rank)
    return [(b, p, g) for b in BACKENDS for p in LOADS]


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name):
    """dram bytes per launch of `name` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                k, _, v = line.partition(":")
                if k.strip() == name:
                    return float(v.split()[0])
    except OSError:
        pass
    return None


# ---- our arm ----------------------------------------------------------------------
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import aspher_b200 as asb
    from aspher_b200 import _lib

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=dev)
    Ns = args.ns
    N = Ns * Ns
    probs = problem_gaps(Ns, rank)
    ops = {b: asb.Operator(b, Ns) for b in BACKENDS}
    gdev = {id(g): torch.from_numpy(g).to(dev) for (_, _, g) in probs}
    gpin = {id(g): torch.from_numpy(g).pin_memory() for (_, _, g) in probs}
    pin_out = torch.empty(N, dtype=torch.float64).pin_memory()
    pout = torch.empty(N, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def step_mixed():
        res = []
        for (b, p, g) in probs:
            r, rf = asb.solve_device_mixed(ops[b], gdev[id(g)], p, tol=TOL, polish=True,
                                           precond="fourier", light=True, pressure_out=pout)
            res.append((r, rf))
        return res

    def step_fp64():
        res = []
        for (b, p, g) in probs:
            res.append(asb.solve_device(ops[b], gdev[id(g)], p, tol=TOL, precond="fourier",
                                        dtype=torch.float64, light=True, pressure_out=pout))
        return res

    solvers = {b: asb.ContactSolver(Ns, backend=b) for b in BACKENDS}

    def step_e2e():
        for (b, p, g) in probs:
            r = solvers[b].solve(gpin[id(g)], p, tol=TOL, precond="fourier",
                                 precision="float_then_double")
            pin_out.copy_(r.pressure_device, non_blocking=True)
            torch.cuda.current_stream().synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        out = None
        for _ in range(steps):
            flush.zero_()
            out = fn()
        e1.record()
        barrier()
        wall = time.perf_counter() - t0
        dt = e0.elapsed_time(e1) / 1e3
        if world > 1:
            t = torch.tensor([dt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        return dt, wall, out

    # accuracy gate (outside the timed region): mixed vs plain FP64
    gate = []
    for (b, p, g) in probs:
        rm, rf = asb.solve_device_mixed(ops[b], gdev[id(g)], p, tol=TOL, precond="fourier",
                                        light=True)
        rd = asb.solve_device(ops[b], gdev[id(g)], p, tol=TOL, precond="fourier",
                              dtype=torch.float64, light=True)
        pm, pd = rm.pressure, rd.pressure
        rel = float(np.linalg.norm(pm - pd) / np.linalg.norm(pd))
        gate.append(dict(backend=b, p_nominal=p, status=rm.status, fp64_status=rd.status,
                         iterations=rm.iterations, float_iterations=rf.iterations,
                         fp64_iterations=rd.iterations, pressure_rel_l2=rel,
                         d_contact_area=abs(rm.contact_area - rd.contact_area),
                         contact_area=rm.contact_area))
    ok = all(x["status"] == "converged" and x["pressure_rel_l2"] <= 10 * TOL and
             x["d_contact_area"] <= 1e-4 for x in gate)

    for _ in range(args.warmup):
        step_mixed()
    bus = None
    try:
        pr = torch.cuda.get_device_properties(dev)
        bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
    except Exception:
        bus = None
    clk = ClockSampler(bus)
    clk.start()
    l0 = _lib.lib().aspher_launch_count()
    dt, wall, last = timed(step_mixed, args.steps)
    launches = int(_lib.lib().aspher_launch_count() - l0)
    clocks = clk.stop()
    n_solves = len(probs) * args.steps * world
    value = n_solves / dt
    iters = [r.iterations for r, _ in last]

    # plain FP64 GPU comparator
    for _ in range(1):
        step_fp64()
    dt64, _, last64 = timed(step_fp64, max(1, args.steps // 2))
    value64 = len(probs) * max(1, args.steps // 2) * world / dt64

    # end to end through the public API (pinned H2D of the gap, D2H of p)
    step_e2e()
    dte, _, _ = timed(step_e2e, args.steps)
    value_e2e = n_solves / dte

    # roofline: the operator apply (row_fwd + col + row_inv), FP32, Ns=2048,
    # free space, timed with CUDA events on the launching stream
    peak, peak_kind = measured_peak()
    op = ops["fft"]
    xs = [torch.randn(N, dtype=torch.float32, device=dev) for _ in range(2)]
    ys = torch.empty(N, dtype=torch.float32, device=dev)
    for i in range(3):
        op.matvec_(xs[i % 2], ys)
    torch.cuda.synchronize()
    ts = []
    for i in range(20):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        c = torch.cuda.Event(enable_timing=True)
        a.record()
        op.matvec_(xs[i % 2], ys)
        c.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(c) / 1e3)
    t_apply = statistics.mean(ts)
    alg_bytes = 12 * 4 * N  # 12 b N, b = 4 (free-space apply model)
    achieved = alg_bytes / t_apply / 1e9

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64",
            "data": "synthetic (seeded self-affine surfaces)",
            "config": {"workload": "Ns=2048 single solves: fft+periodic x p_nominal "
                                   "{0.001,0.005,0.02}, tol 1e-6, stencil precond, "
                                   "FP32 CG + FP64 polish", "grid_size": Ns,
                       "solves_per_step_per_gpu": len(probs), "tol": TOL,
                       "l2": "256 MB buffer written between steps; working set "
                             "> 126 MB L2"},
            "fp64_gpu": {"value": value64, "unit": "solves/s",
                         "ratio_mixed_over_fp64": value / value64,
                         "iterations": [r.iterations for r in last64]},
            "iterations": iters,
            "accuracy_gate": {"pass": ok, "problems": gate},
            "e2e": {"value": value_e2e, "unit": "solves/s",
                    "h2d_bytes_per_step": 8 * N * len(probs),
                    "d2h_bytes_per_step": 8 * N * len(probs)},
            "roofline": {"bound": "hbm", "kernel": "free-space apply FP32 Ns=2048 "
                         "(row_fwd+col+row_inv)", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profiled_traffic("fft_apply_f32_2048"),
                         "alg_bytes": alg_bytes, "t_apply_ms": t_apply * 1e3},
            "gpu_launches": launches,
            "clocks": clocks,
            "wall_s_timed": wall,
        }
        it64 = [r.iterations for r in last64]
        line["cpu_baseline"] = (cpu_baseline(gpu_fp64_iterations=it64[1])
                                if not os.environ.get("BENCH_SKIP_CPU")
                                else {"value": None, "sample": "skipped (BENCH_SKIP_CPU)"})
        print(json.dumps(line), flush=True)
    for b in list(ops):
        del ops[b]
    if world > 1:
        dist.destroy_process_group()


# ---- CPU baseline / reference arm (the oracle restatement) ----------------------------
def _oracle_iterations():
    with open(os.path.join(ROOT, "tests", "golden", "bench_iterations.json")) as f:
        return json.load(f)["problems"]


def _oracle_sample(backend, pbar, g, n_iter):
    """Seconds per PCG iteration of the oracle on one problem (n_iter iterations)."""
    from oracle.api import ContactSolver
    s = ContactSolver(NS, backend=backend)
    t0 = time.perf_counter()
    r = s.solve(g, pbar, tol=TOL, max_iter=n_iter, precond="fourier")
    dt = time.perf_counter() - t0
    return dt / max(1, r.iterations), r.iterations


def cpu_baseline(n_iter=6, gpu_fp64_iterations=None):
    """Oracle FP64 solve of one problem (fft, p=0.005), n_iter iterations timed,
    scaled to that problem's full oracle iteration count (or, when that count
    is not recorded, to the FP64 GPU solve's count for the same problem)."""
    try:
        from aspher_b200.surfaces import self_affine_gap
        from oracle import operators as oops
        g = self_affine_gap(NS, hurst=0.8, rms=0.002, seed=SEED)
        try:
            full = _oracle_iterations()["fft_0.005"]["iterations"]
        except (OSError, KeyError):
            full = gpu_fp64_iterations
        if not full:
            raise RuntimeError("no iteration count to scale the sample by")
        spi, k = _oracle_sample("fft", 0.005, g, n_iter)
        return {"value": 1.0 / (spi * full), "unit": "solves/s", "cores": oops.WORKERS,
                "kind": "port",
                "sample": "oracle FP64 solve, fft Ns=2048 p=0.005 stencil precond: %d PCG "
                          "iterations timed (%.2f s/iteration), scaled to the oracle's full "
                          "%d iterations; scipy pocketfft on %d threads, numpy vector passes "
                          "single-threaded" % (k, spi, full, oops.WORKERS)}
    except Exception as e:  # the baseline must never sink the GPU line
        return {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                "sample": "unavailable: %s" % e}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from aspher_b200.surfaces import self_affine_gap
    from oracle import operators as oops
    g = self_affine_gap(NS, hurst=0.8, rms=0.002, seed=SEED)
    its = _oracle_iterations()
    probs = [(b, p) for b in BACKENDS for p in LOADS]
    n_iter = 4
    for w in range(args.warmup):
        b, p = probs[w % len(probs)]
        _oracle_sample(b, p, g, 1)
    per_solve = []
    t0 = time.perf_counter()
    for s in range(args.steps):
        b, p = probs[s % len(probs)]
        spi, _ = _oracle_sample(b, p, g, n_iter)
        per_solve.append(spi * its["%s_%g" % (b, p)]["iterations"])
    wall = time.perf_counter() - t0
    sec = statistics.mean(per_solve)
    value = 1.0 / sec
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": sec * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded self-affine surfaces)",
        "config": {"workload": "Ns=2048 single solves: fft+periodic x p_nominal "
                               "{0.001,0.005,0.02}, tol 1e-6, stencil precond",
                   "grid_size": NS, "tol": TOL},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": oops.WORKERS,
                         "kind": "port",
                         "sample": "per step: %d oracle FP64 PCG iterations of one problem "
                                   "(cycling the 6), scaled by its full oracle iteration "
                                   "count" % n_iter},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s_timed": wall,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
