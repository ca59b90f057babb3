"""CPU, world_size 2 over gloo: the multi-rank path of a sharded ensemble.

Ensembles shard by instance with no exchange in the data path; the only
collectives are one sum and one max all-reduce of the throughput
(heom_b200.reduce_throughput) and, for observables, a sum of per-rank population
traces.  Here each rank propagates its shard of a small ensemble with the
oracle on the CPU and the reduced results must equal a single-process run."""
import os
import socket

import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


SYSTEMS = [(3, 2, 1, 1), (4, 2, 1, 2), (3, 3, 2, 3), (5, 1, 1, 4), (4, 3, 1, 5)]  # (sites, depth, M, seed)


def ensemble_pops(indices):
    """Sum over the given instances of the final site-0 populations, and their ADO-steps."""
    tot, ados = 0.0, 0
    for k in indices:
        n, d, m, seed = SYSTEMS[k]
        prob = ho.build_problem(ho.drude_system(n, d, m, seed=seed))
        _, pops = ho.propagate(prob, 1e-15, 20, 20, threads=1)
        tot += pops[-1][0]
        ados += prob.graph.nodes * 20
    return tot, ados


def worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [ho.build_graph(n * m, d).nodes * n * n for n, d, m, _ in SYSTEMS]
    mine = hb.shard_instances(sizes, world, rank)
    pop_sum, ados = ensemble_pops(mine)
    t = torch.tensor([pop_sum], dtype=torch.float64)
    dist.all_reduce(t)
    job_ados, job_secs = hb.reduce_throughput(dist, ados, 1.0 + rank, "cpu")
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out.put((float(t.item()), job_ados, job_secs, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_covers_every_instance_once_and_balances():
    sizes = [int(x) for x in np.random.default_rng(3).integers(1, 1000, size=64)]
    for world in (1, 2, 3, 8):
        parts = [hb.shard_instances(sizes, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = [sum(sizes[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)  # greedy largest-first bound


def test_two_rank_gloo_ensemble_matches_one_process():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    pop_sum, job_ados, job_secs, gathered = q.get(timeout=10)
    ref_sum, ref_ados = ensemble_pops(range(len(SYSTEMS)))
    assert sorted(gathered[0] + gathered[1]) == list(range(len(SYSTEMS)))
    assert abs(pop_sum - ref_sum) <= 1e-14
    assert job_ados == ref_ados
    assert job_secs == 2.0  # the slowest rank
