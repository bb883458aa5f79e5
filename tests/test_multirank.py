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


def test_seed_shards_cover_every_seed():
    from phix_b200.surrogate import dp_update_counts, shard_seeds
    shards = [shard_seeds(range(100, 300), r, 3) for r in range(3)]
    assert sorted(s for x in shards for s in x) == list(range(100, 300))
    assert sorted(len(x) for x in shards) == [66, 67, 67]
    # 801 snapshots, chunks of 25 trajectories, batch 16, 2 epochs
    counts = dp_update_counts([len(x) for x in shards], 801, 25, 16, 2)
    assert counts[0] == counts[1] > counts[2]
    assert counts[2] == 2 * ((25 * 800) // 16) * 2 + 2 * ((16 * 800) // 16)


def _dp_active_worker(rank, world, port, out):
    _init(rank, world, port)
    try:
        from phix_b200 import surrogate as S
        g = torch.full((5,), float(rank + 1), dtype=torch.float64)
        S.allreduce_active_mean_(g, active=(rank == 0), n_active=1)  # rank 1's shard is used up
        both = torch.full((5,), float(rank + 1), dtype=torch.float64)
        S.allreduce_active_mean_(both, active=True, n_active=2)
        got = [None] * world
        dist.all_gather_object(got, (g.numpy().copy(), both.numpy().copy()))
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


def test_padded_update_takes_only_the_active_ranks_gradient():
    got = _run(_dp_active_worker)
    for g, both in got:  # every rank applies the same averaged gradient
        assert np.array_equal(g, np.full(5, 1.0))
        assert np.array_equal(both, np.full(5, 1.5))


def _bench_worker(rank, world, port, out):
    _init(rank, world, port)
    try:
        import bench
        env = {"WORLD_SIZE": str(world), "RANK": str(rank)}
        w = bench.resolve_world(world, env)
        # rank r timed (r + 1) * 10 ms and advanced (r + 1) * 1000 cells per time step
        total_ms, cells, e2e_ms = bench.combine_over_ranks(10.0 * (rank + 1), 1000.0 * (rank + 1),
                                                           3.0 + rank, torch.device("cpu"), w)
        job = bench.job_summary(w, 4, 100, total_ms, cells)
        if rank == 0:
            out.put((job, e2e_ms))
    finally:
        dist.destroy_process_group()


def test_bench_rank_logic_two_ranks():
    job, e2e_ms = _run(_bench_worker)
    assert job["n_gpus"] == 2
    assert job["ms_per_step"] == 20.0 / 4  # the slowest rank
    assert job["value"] == 3000.0 * 100 * 4 / 0.020  # cells of both ranks
    assert e2e_ms == 4.0


def test_bench_world_size_must_match_gpus():
    import bench
    assert bench.resolve_world(1, {}) == 1
    assert bench.resolve_world(4, {}) == 1  # main() launches the ranks itself
    assert bench.resolve_world(2, {"WORLD_SIZE": "2"}) == 2
    with pytest.raises(SystemExit):
        bench.resolve_world(4, {"WORLD_SIZE": "2"})
    cmd = bench.launcher_command(["--gpus", "2", "--steps", "3"], 2, 29512)
    assert "--nproc-per-node=2" in cmd and "--master-addr=127.0.0.1" in cmd
    assert cmd[-4:] == ["--gpus", "2", "--steps", "3"]


def test_data_parallel_gradient_average_equals_full_batch():
    avg, full = _run(_dp_worker)
    assert np.allclose(avg, full, rtol=1e-9, atol=1e-12 * np.abs(full).max())
