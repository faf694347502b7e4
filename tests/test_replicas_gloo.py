"""The multi-GPU path of the bench is N independent replicas: no collective
on the data path, a barrier around the timed region and the max over ranks
of the device time.  Its host side (bench.barrier, bench.allreduce_max) runs
here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import sys

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench

        bench.barrier(world)
        ms = bench.allreduce_max(times[rank], world, None)
        bench.barrier(world)
        # the whole-job value: every rank's solves over the slowest rank's time
        steps = 10
        out[rank] = (ms, world * steps / (ms / 1e3))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_replicas_report_the_slowest_rank():
    world, times = 2, [37.5, 41.25]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, times, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0] == res[1]
    ms, value = res[0]
    assert ms == max(times)
    assert value == pytest.approx(world * 10 / (max(times) / 1e3))


def test_single_rank_needs_no_process_group():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    bench.barrier(1)
    assert bench.allreduce_max(3.5, 1, None) == 3.5
