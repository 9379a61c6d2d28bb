"""The multi-GPU path is replicas only: every rank bounds its own boxes and the only collective
is the max over ranks of the timing. Two gloo ranks on the CPU check that the ranks' boxes
are distinct, that the max-over-ranks reduction is what bench.py reports, and that bounding
each rank's shard separately (the oracle stands in for the device) equals bounding the union
in one process: the partition changes nothing."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from gear_b200 import graph, problems
        from oracle.crown import CrownOracle
        lo, hi = bench.rank_boxes("quad_exp_n10", 6, rank)
        g = graph.trace(problems.make_instance("quad_exp_n10", 0), lo[:2])
        lb = CrownOracle(g).compute_bounds(lo.numpy(), hi.numpy())[0]
        slowest = bench.max_over_ranks(10.0 + rank, world, torch.device("cpu"))
        gathered = [None] * world
        dist.all_gather_object(gathered, (lo.numpy(), hi.numpy(), lb, slowest))
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = out.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (lo0, hi0, lb0, s0), (lo1, hi1, lb1, s1) = res
    assert s0 == s1 == 11.0                      # the max over ranks
    assert not np.allclose(lo0, lo1)             # each rank has its own boxes
    from gear_b200 import graph, problems
    from oracle.crown import CrownOracle
    g = graph.trace(problems.make_instance("quad_exp_n10", 0), torch.tensor(lo0[:2]))
    lb = CrownOracle(g).compute_bounds(np.concatenate([lo0, lo1]), np.concatenate([hi0, hi1]))[0]
    assert np.array_equal(lb, np.concatenate([lb0, lb1]))
