"""The multi-GPU form of bench.py is N independent replicas (one field per rank,
no collective on the data path); only the whole-job aggregates cross ranks:
times take the max over the ranks, counts the sum.  Those host steps run here as
two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path[:0] = [ROOT, os.path.join(ROOT, "crowdphot.jl_b200")]
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        mx, sm = bench.max_and_sum_over_ranks([1.5 * (rank + 1), 10 * (rank + 1), 7], "cpu")
        q.put((rank, mx, sm, bench.replica_seed(1002, rank)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    for rank, mx, sm, seed in got:
        assert mx == [3.0, 20.0, 7.0]  # the slowest replica's time; the per-rank maxima
        assert sm == [4.5, 30.0, 14.0]  # counts summed over the job
    assert got[0][3] != got[1][3]  # every replica fits its own field


def test_single_process_aggregate_is_identity():
    sys.path[:0] = [ROOT, os.path.join(ROOT, "crowdphot.jl_b200")]
    import bench
    mx, sm = bench.max_and_sum_over_ranks([2.0, 5, 1])
    assert mx == sm == [2.0, 5.0, 1.0]
