"""The multi-GPU form of the benchmark is replicas only (each rank advances
its own torus, no data-path collective); its host logic -- maximum over
ranks of the timed region and the whole-job aggregate -- runs here as two
gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank           # rank 1 is the slow one
    m = bench.max_over_ranks(ms, dist, "cpu")
    rate = bench.aggregate_rate(world, 512 * 512, m * 1e-3)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, m, rate))


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in res] == [15.0, 15.0]
    assert res[0][2] == pytest.approx(2 * 512 * 512 / 15e-3)
