"""The multi-GPU plumbing of bench.py, on CPU: the path does not shard, so N ranks are N
independent replicas whose only collectives are a barrier and the max over ranks of the timed
region. 2 gloo ranks on 127.0.0.1 run the same steps as the NCCL ranks of `bench.py --gpus N`."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    dist, barrier, max_over_ranks = bench._plumbing(world, backend="gloo")
    try:
        barrier()
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
        ms_max = max_over_ranks(ms)
        out[rank] = (ms_max, bench.replica_value(world, 1000, 4, ms_max))
        barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    # Both ranks see the max (15 ms); the whole job did 2 x 1000 x 4 units in 15 ms.
    for rank in range(world):
        ms_max, value = got[rank]
        assert ms_max == 15.0
        assert value == pytest.approx(2 * 1000 * 4 / 0.015)
