"""Multi-process path of bench.py on the CPU (gloo, 2 ranks): every rank
times its own replica and the job reports the slowest rank's time; the
value counts all ranks' points."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    r, w, local = bench.dist_info()
    dist.init_process_group("gloo", rank=r, world_size=w,
                            timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 + 5.0 * r, dist, "cpu")
    out.put((r, w, local, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
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
    assert [(r, w, l) for r, w, l, _ in res] == [(0, 2, 0), (1, 2, 1)]
    assert all(ms == pytest.approx(15.0) for *_, ms in res)


def test_single_process_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
