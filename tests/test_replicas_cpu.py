"""The multi-GPU path of bench.py on CPU: world_size 2 over gloo. Ranks step
disjoint scene sets (replicas, no collective on the data path); the job's
time is the maximum over ranks."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "threejs-particle-fluids_b200")]
    import bench
    from pfsim import workloads as W

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks([10.0 + rank, 5.0 - rank], "cpu")
        recipes = W.batch_stream(6, seed=bench.replica_seed(rank))
        names = [r.name for r in recipes]
        gathered = [None] * world
        dist.all_gather_object(gathered, names)
        # the job's units are every replica's own (its scenes differ)
        mine = sum(r.particle_substeps for r in recipes)
        total = bench.sum_over_ranks(mine, "cpu")
        out.put((rank, ms, gathered, mine, total))
    finally:
        dist.destroy_process_group()


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mine = {rank: m for rank, _, _, m, _ in res}
    for rank, ms, gathered, _, total in res:
        assert ms == [11.0, 5.0]  # max over ranks, element-wise
        assert gathered[0] != gathered[1]  # each rank its own scenes
        assert total == mine[0] + mine[1]
