"""Uneven batches: grouping, the multi-GPU partition, and (GPU) parity.

The partition of problems across ranks is host logic (no collective on the
data path); its N > 1 path is exercised with two gloo ranks on the CPU.
"""

import os

import numpy as np
import pytest

from aspher_b200.batch import lpt_partition, solve_cost, uneven_problems


def test_uneven_workload_is_seeded_and_mixed():
    a = uneven_problems()
    b = uneven_problems()
    assert a == b and len(a) == 96
    sizes = [p["grid_size"] for p in a]
    assert set(sizes) <= {256, 512, 1024, 2048} and len(set(sizes)) == 4
    assert [p["backend"] for p in a[:4]] == ["fft", "periodic", "fft", "periodic"]
    assert all(1e-3 <= p["p_nominal"] <= 2e-2 for p in a)
    assert all(0.6 <= p["hurst"] <= 0.9 for p in a)
    assert [p["seed"] for p in a[:3]] == [1000, 1001, 1002]


@pytest.mark.parametrize("nbins", [1, 2, 3, 8])
def test_lpt_partition_is_complete_disjoint_and_balanced(nbins):
    probs = uneven_problems()
    costs = [solve_cost(p["backend"], p["grid_size"]) for p in probs]
    bins = lpt_partition(costs, nbins)
    flat = sorted(i for b in bins for i in b)
    assert flat == list(range(len(probs)))
    loads = [sum(costs[i] for i in b) for b in bins]
    # LPT bound: max load <= mean load + the largest single job
    assert max(loads) <= sum(costs) / nbins + max(costs) + 1e-9


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    probs = uneven_problems(n=40, seed=5)
    costs = [solve_cost(p["backend"], p["grid_size"]) for p in probs]
    mine = lpt_partition(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_partition_across_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = q.get(timeout=120)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = got
    assert not set(a) & set(b)
    assert sorted(a + b) == list(range(40))


@pytest.mark.gpu
def test_solve_many_matches_single_solves():
    torch = pytest.importorskip("torch")
    from aspher_b200 import Operator, solve_device_mixed
    from aspher_b200.batch import problem_gap, solve_many
    probs = uneven_problems(n=10, seed=9, sizes=(64, 128), weights=(0.5, 0.5))
    gaps = [problem_gap(p) for p in probs]
    rs = solve_many(probs, gaps, tol=1e-6, polish_tol=1e-7)
    torch.cuda.synchronize()
    for p, g, r in zip(probs, gaps, rs):
        assert r.status == "converged", (p, r.status)
        op = Operator(p["backend"], p["grid_size"])
        r1, _ = solve_device_mixed(op, torch.as_tensor(g, device="cuda"), p["p_nominal"],
                                   tol=1e-6, polish_tol=1e-7, light=True)
        a, b = r.pressure.ravel(), r1.pressure.ravel()
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)
        assert abs(r.contact_area - r1.contact_area) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "float", "float_then_double"])
def test_solve_many_c_abi_mixed_grid_sizes(precision):
    """aspher_solve_many through the C ABI on problems of four grid sizes and
    both backends (and two domain sizes): every problem certified, each
    result equal to that problem's own solve of the same precision, the
    serial and concurrent forms agree, and groups and problems come back in
    input order."""
    torch = pytest.importorskip("torch")
    import aspher_b200 as asb
    from aspher_b200.batch import problem_gap, solve_many
    probs = uneven_problems(n=12, seed=11, sizes=(32, 64, 128, 256),
                            weights=(0.25, 0.25, 0.25, 0.25))
    probs[3]["domain_size"] = 2.0
    gaps = [problem_gap(p) for p in probs]
    tol = 1e-6 if precision != "double" else 1e-8
    kw = dict(tol=tol, precision=precision)
    rs = solve_many(probs, gaps, **kw)
    rs_serial = solve_many(probs, gaps, concurrent=False, **kw)
    torch.cuda.synchronize()
    for i, (p, g, r, rz) in enumerate(zip(probs, gaps, rs, rs_serial)):
        assert r.status == "converged", (i, p, r.status)
        assert r.pressure.shape == (p["grid_size"], p["grid_size"])
        op = asb.Operator(p["backend"], p["grid_size"], p.get("domain_size", 1.0))
        gd = torch.as_tensor(g, device="cuda")
        if precision == "double":
            r1 = asb.solve_device(op, gd, p["p_nominal"], tol=tol, precond="fourier",
                                  dtype=torch.float64, light=True, keep_best=False)
        else:
            r1, _ = asb.solve_device_mixed(op, gd, p["p_nominal"], tol=tol, precond="fourier",
                                           polish=precision == "float_then_double",
                                           light=True, keep_best=False)
        a, b = r.pressure.ravel(), r1.pressure.ravel()
        assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b), (i, p)
        assert np.array_equal(r.pressure, rz.pressure), i
        assert r.iterations == r1.iterations == rz.iterations, i


@pytest.mark.gpu
def test_solve_many_rejects_bad_problems():
    pytest.importorskip("torch")
    from aspher_b200.batch import solve_many
    probs = [dict(backend="fft", grid_size=64, p_nominal=0.01),
             dict(backend="periodic", grid_size=64, p_nominal=0.01),
             dict(backend="fft", grid_size=64, p_nominal=-1.0)]
    gaps = [np.zeros(64 * 64)] * 3
    with pytest.raises(ValueError, match="problem 2"):
        solve_many(probs, gaps)
    with pytest.raises(ValueError, match="polish_tol"):
        solve_many(probs[:2], gaps[:2], tol=1e-6, polish_tol=1e-5)
