"""The multi-GPU path of bench.py is replicas only (the sweep, the hydro step and the
scattering of the benchmark workloads run on one GPU; no data-path collective):
each rank times its own replica and the job time is the maximum over ranks.  This
checks that host logic with two gloo ranks on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (ws, rank, rank)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        job = bench.max_over_ranks(ms, ws, "cpu")
        value = bench.job_throughput(1000, ws, 4, job)
        out.put((rank, job, value))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(90)
    assert all(p.exitcode == 0 for p in ps)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, job, value in res:
        assert job == 15.0  # the slower replica sets the job time on every rank
        assert value == 2 * 1000 * 4 / 0.015  # whole-job units/s over both replicas
