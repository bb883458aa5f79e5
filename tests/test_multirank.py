"""The N > 1 paths on CPU: two gloo ranks in separate processes.

* Batched configuration: the job of 2 x 64 independent instances is split
  across the ranks by phix_b200.workloads.partition_instances (no collective on
  the data path); every instance is owned by exactly one rank and the loads
  are balanced to within one instance.
* Surrogate data-parallel training: each rank computes the gradient of its
  half of a batch (the numpy oracle stands in for the GPU kernels, which the
  CPU cannot run), phix_b200.surrogate.allreduce_mean_ averages them, and the
  result equals the gradient of the whole batch.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _batch_worker(rank, world, port, out):
    _init(rank, world, port)
    try:
        from phix_b200 import workloads
        grids, *_ = workloads.ch2d_batch(ninst=64 * world)
        costs = [g.n[0] * g.n[1] for g in grids]
        mine = workloads.partition_instances(costs, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, (mine, sum(costs[i] for i in mine)))
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


def _dp_worker(rank, world, port, out):
    _init(rank, world, port)
    try:
        from oracle import surrogate_oracle as so
        from phix_b200 import surrogate as S
        params = so.init_params(3)
        params[6] = params[6] * 10.0
        rng = np.random.default_rng(7)
        c = rng.uniform(0.3, 0.7, size=(4, 8, 16))
        cn = c + 0.01 * rng.standard_normal(c.shape)
        half = slice(2 * rank, 2 * rank + 2)
        o, cache = so.forward(params, c[half], 0.5, 4.0)
        _, do = so.mse_loss_and_grad(o, (cn[half] - c[half]) / 0.01)
        flat = lambda gs: np.concatenate([np.asarray(x, np.float64).ravel() for x in gs])
        g = torch.from_numpy(flat(so.backward(params, cache, do)))
        S.allreduce_mean_(g)
        if rank == 0:
            o, cache = so.forward(params, c, 0.5, 4.0)
            _, do = so.mse_loss_and_grad(o, (cn - c) / 0.01)
            full = flat(so.backward(params, cache, do))
            out.put((g.numpy(), full))
    finally:
        dist.destroy_process_group()


def _run(worker, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    return res


def test_batch_instances_partitioned_across_two_ranks():
    got = _run(_batch_worker)
    owned = sorted(i for mine, _ in got for i in mine)
    assert owned == list(range(128))
    loads = [load for _, load in got]
    assert max(loads) - min(loads) <= 1024 * 1024  # within the largest instance


def test_seed_shards_are_disjoint_and_equal_sized():
    from phix_b200.surrogate import shard_seeds
    shards = [shard_seeds(range(100, 300), r, 3) for r in range(3)]
    assert len({len(x) for x in shards}) == 1
    flat = [s for x in shards for s in x]
    assert len(flat) == len(set(flat)) == 198


def test_data_parallel_gradient_average_equals_full_batch():
    avg, full = _run(_dp_worker)
    assert np.allclose(avg, full, rtol=1e-9, atol=1e-12 * np.abs(full).max())
