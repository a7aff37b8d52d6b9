"""The multi-GPU path's host logic on CPU: two gloo ranks shard a batch of
uneven horizons, solve their instances (with the CPU oracle standing in for the
GPU solve), and the gathered results equal one process solving the whole batch;
the adjoint's weight-gradient all-reduce equals one process summing the whole
batch; the timing reduction takes the max over ranks."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NS = [6, 12, 4, 9, 12, 5, 8]
CFG = dict(dt=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)


def solve_instances(ids):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import importlib
    import oracle_py as O
    P = importlib.import_module("gpu-pcg-tracking_b200.problem")
    par = O.make_params(dt=CFG["dt"], integrator=CFG["integrator"], qd_cost=CFG["qd_cost"], r_cost=CFG["r_cost"])
    sol = O.make_solver(linsys=2, sqp_max_iter=3)
    out = {}
    for i in ids:
        p = P.make_problem(NS[i], i, dt=CFG["dt"])
        xu, lam, rho, st, _ = O.sqp_solve(par, sol, NS[i], p["goal"], p["lam"], p["xu"], 1e-3)
        out[i] = (np.asarray(xu), float(rho))
    return out


def weight_grads(ids):
    """Deterministic stand-ins for gpt_sqp_adjoint's per-instance weight gradients of instances ids."""
    ids = list(ids)
    gq = torch.tensor([[np.sin(i + 0.1 * j) for j in range(7)] for i in ids], dtype=torch.float32)
    gr = torch.tensor([[np.cos(i - 0.2 * j) for j in range(7)] for i in ids], dtype=torch.float32)
    ge = torch.tensor([0.5 + i for i in ids], dtype=torch.float32)
    return gq, gr, ge


def worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import importlib
    shard = importlib.import_module("gpu-pcg-tracking_b200.shard")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ids = shard.shard_instances(NS, rank, world)
    res = solve_instances(ids)
    gathered = [None] * world
    dist.all_gather_object(gathered, {"ids": ids, "res": res})
    tmax = shard.max_over_ranks(float(rank + 1), device="cpu")
    # the adjoint's weight-gradient exchange: every rank contributes its instances' gradients
    gq, gr, ge = weight_grads(ids)
    packed = shard.allreduce_weight_grads(gq, gr, ge)
    if rank == 0:
        q.put({"gathered": gathered, "tmax": tmax, "grads": packed.numpy()})
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_partition_is_complete_and_balanced(gpt):
    import importlib
    shard = importlib.import_module("gpu-pcg-tracking_b200.shard")
    mixed = [32, 64, 128, 256, 32, 64, 128, 256, 64, 32]
    for world in (1, 2, 3, 4):
        parts = [shard.shard_instances(mixed, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(mixed)))
        loads = [sum(mixed[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(mixed), (world, loads)
    assert shard.weak_scaling_ids(1, 2, 3) == [3, 4, 5]
    assert shard.max_over_ranks(2.5) == 2.5  # no process group: the value itself
    with pytest.raises(ValueError):
        shard.shard_instances(mixed, 2, 2)


def test_two_gloo_ranks_equal_one_process(gpt, oracle):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out["tmax"] == 2.0
    # the all-reduced weight gradient equals one process summing the whole batch
    gq, gr, ge = weight_grads(range(len(NS)))
    want = torch.cat([gq.sum(0), gr.sum(0), ge.sum().reshape(1)]).to(torch.float64).numpy()
    np.testing.assert_allclose(out["grads"], want, rtol=1e-6, atol=1e-6)
    ids = sorted(i for g in out["gathered"] for i in g["ids"])
    assert ids == list(range(len(NS)))
    merged = {}
    for g in out["gathered"]:
        merged.update(g["res"])
    whole = solve_instances(range(len(NS)))
    for i in range(len(NS)):
        np.testing.assert_array_equal(merged[i][0], whole[i][0])
        assert merged[i][1] == whole[i][1]
