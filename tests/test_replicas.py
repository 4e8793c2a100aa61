"""The multi-GPU form of the bench is replicas only: each rank steps its own copy of the workload
and the job reports the summed particle-steps over the slowest rank's time.  This checks that
reduction over two gloo ranks on the CPU (no GPU, no collective on the data path)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))  # fmt: skip
    import bench

    ms, total = bench.combine_ranks(10.0 * (rank + 1), 1000 * (rank + 1), "cpu")
    out[rank] = (ms, total)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_timing_is_max_over_ranks_and_work_is_summed():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    assert dict(out) == {0: (20.0, 3000.0), 1: (20.0, 3000.0)}

