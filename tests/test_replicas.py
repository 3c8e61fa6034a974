"""Replica path of bench.py --gpus N on CPU: two gloo ranks on 127.0.0.1.

Each rank reports a different timed region; both must see the maximum, and the
whole-job rate must count the units of every rank against that maximum.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    from stda_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    replicas.barrier(dist)
    seconds = 1.0 + rank          # rank 1 is the slower one
    mx = replicas.max_over_ranks(dist, seconds)
    rate = replicas.whole_job_rate(10, world, mx)
    replicas.barrier(dist)
    dist.destroy_process_group()
    out.put((rank, mx, rate))


def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.0, 2.0]
    assert all(abs(r[2] - 10.0) < 1e-12 for r in res)   # 2 ranks x 10 units / 2 s


def test_single_process_without_a_group():
    from stda_b200 import replicas
    assert replicas.max_over_ranks(None, 3.5) == 3.5
    replicas.barrier(None)
    assert replicas.whole_job_rate(5, 1, 0.5) == pytest.approx(10.0)
