"""The replica (multi-GPU) path of bench.py on CPU: two gloo ranks reduce
their timings to the slowest rank's time and the sum of their work, and the
reference arm does its work on rank 0 only."""
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


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    t, w = bench.reduce_over_ranks(dist, 1.0 + rank, 100.0 * (rank + 1), "cpu")
    out[rank] = (t, w)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_max_time_and_total_work():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1] == (2.0, 300.0)


def test_single_process_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(None, 1.5, 7.0, "cpu") == (1.5, 7.0)


def test_reference_arm_other_ranks_do_no_work(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        workload = "mars"
        steps = 1
        warmup = 0

    bench.run_reference(A(), rank=1, world=2)
    assert capsys.readouterr().out == ""
