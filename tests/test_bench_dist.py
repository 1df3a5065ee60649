"""CPU test of the multi-rank plumbing bench.py uses with --gpus N (one
process per GPU under torchrun): ranks optimise disjoint queries, the timed
region is reduced as the maximum over ranks, and the whole-job value divides
all ranks' queries by that maximum.  Two gloo ranks on 127.0.0.1."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seeds = bench.rank_seeds(rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        mx = bench.max_over_ranks(10.0 + rank, dist, "cpu")
        out.put((rank, gathered, mx, bench.whole_job_ms_per_query(mx, 4, world)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_queries_and_take_the_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, mx, value in res:
        assert set(gathered[0]).isdisjoint(gathered[1])      # weak scaling: different queries
        assert len(gathered[0]) == len(gathered[1])
        assert mx == 11.0                                     # the slower rank's time
        assert value == 11.0 / 8                              # 2 ranks x 4 steps
