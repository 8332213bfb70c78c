"""Multi-GPU plumbing on two gloo ranks (CPU): bench.py's rank-distinct
replica sets (weak scaling, no data exchange), job totals summed over ranks,
job time = max over ranks; and the end-of-run collection of per-replica
results (gather.py) with uneven replica counts per rank."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    reps = bench.rank_replicas(6, 2024, rank)
    n_local = sum(sum(r["initial_populations"].values()) for r in reps)
    total = bench.job_particle_steps(n_local, world, 100)
    slowest = bench.max_over_ranks(1.0 + rank, world)
    seeds = [r["random_seed"] for r in reps]
    q.put((rank, n_local, total, slowest, seeds))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_weak_scaling_plumbing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, n0, t0, s0, seeds0), (r1, n1, t1, s1, seeds1) = out
    assert set(seeds0).isdisjoint(seeds1), "ranks must run different replicas"
    assert t0 == t1 == (n0 + n1) * 100
    assert s0 == s1 == 2.0


def _gather_worker(rank, world, port, q):
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from flim_microscopy_simulator_with_causal_inference_b200 import gather as G
    R = 3 if rank == 0 else 5  # uneven replica counts
    counters = (np.arange(R * 14, dtype=np.int64).reshape(R, 14) + 1000 * rank)
    tau = np.full((R, 4, 4), 2.0 + rank, dtype=np.float64)
    decay = np.arange(256, dtype=np.int64) * (rank + 1)
    out = G.collect_ensemble(counters, tau, decay)
    q.put((rank, out["counters"], out["tau_maps"], out["decay"]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_collection_of_per_replica_results():
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=240) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_c = np.concatenate([np.arange(3 * 14).reshape(3, 14), np.arange(5 * 14).reshape(5, 14) + 1000])
    want_t = np.concatenate([np.full((3, 4, 4), 2.0), np.full((5, 4, 4), 3.0)])
    want_d = np.arange(256) * 3
    for rank, c, t, d in out:  # every rank holds the whole ensemble in rank order
        assert np.array_equal(c, want_c), rank
        assert np.array_equal(t, want_t), rank
        assert np.array_equal(d, want_d), rank
