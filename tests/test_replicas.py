"""Multi-process host logic of replica runs, on CPU with the gloo backend (world size 2)."""
import os
import socket

import torch.multiprocessing as mp

from pct_reconstruction_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert replicas.world() == (rank, rank, world)
        # rank r took 100 + 50 r ms per step on 1000 histories
        value, ms = replicas.aggregate_throughput(1000, 100.0 + 50.0 * rank)
        out[rank] = (value, ms, replicas.replica_seed(7, rank))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_takes_the_slowest_rank():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    slowest = 150.0
    for rank in range(world):
        value, ms, _ = res[rank]
        assert ms == slowest
        assert abs(value - 2 * 1000 / (slowest / 1000.0)) < 1e-6
    assert res[0][2] != res[1][2]


def test_single_process_is_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    v, ms = replicas.aggregate_throughput(100, 10.0)
    assert ms == 10.0 and abs(v - 10000.0) < 1e-9
