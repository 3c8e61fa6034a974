"""Replica path of bench.py --gpus N on CPU: two gloo ranks on 127.0.0.1.

Each rank reports a different timed region; both must see the maximum, and the
whole-job rate must count the units of every rank against that maximum.  The
split of independent molecules over ranks (shard_by_cost) covers every
molecule exactly once, is the same on every rank, and keeps the loads within
one molecule's cost of each other.
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


def test_shard_by_cost_covers_all_and_balances():
    import numpy as np
    from stda_b200 import replicas
    rng = np.random.default_rng(5)
    costs = rng.integers(1, 1000, size=97).tolist()
    for world in (1, 2, 3, 8):
        parts = replicas.shard_by_cost(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert replicas.shard_by_cost(costs, world) == parts       # deterministic
    assert replicas.shard_by_cost([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        replicas.shard_by_cost([1.0], 0)


def _shard_rank(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    from stda_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    costs = [(7 * k) % 23 + 1 for k in range(40)]
    mine = replicas.shard_by_cost(costs, world)[rank]
    # every rank's share, gathered only to check the split here
    got = [None] * world
    dist.all_gather_object(got, mine)
    done = torch.tensor([float(len(mine))])
    dist.all_reduce(done)
    dist.destroy_process_group()
    out.put((rank, got, int(done.item())))


def test_two_gloo_ranks_split_molecules():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = res[0][1]
    assert res[1][1] == shares                       # the same split on both ranks
    assert sorted(shares[0] + shares[1]) == list(range(40))
    assert not set(shares[0]) & set(shares[1])
    assert res[0][2] == res[1][2] == 40


def _bench_rank(rank, world, port, out):
    import datetime
    import types
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    seen = []

    def fake_server(precision, pool, reqs, arrivals, slots, device, batch=False):
        # stands in for the request server: rank r "takes" 1 + r seconds
        seen.extend(i for i, _, _ in reqs)
        return [], {"makespan_s": 1.0 + rank}

    args = types.SimpleNamespace(batch_pool=3, batch_requests=9, batch_slots=2)
    res = bench.batched_sharded(dist, 0, world, rank, args, dev=None, runner=fake_server)
    dist.destroy_process_group()
    out.put((rank, res, seen))


def test_bench_batched_sharded_on_two_gloo_ranks():
    """bench.py's --gpus N batch path with the server replaced by a fake:
    each rank takes its own share, and the whole-job rate counts every
    request against the slowest rank's time."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, out0, seen0), (r1, out1, seen1) = res
    assert out0["requests_this_rank"] + out1["requests_this_rank"] == 9
    assert out0["slowest_rank_s"] == out1["slowest_rank_s"] == 2.0
    assert out0["solves_per_s"] == pytest.approx(9 / 2.0)
    assert sorted(seen0 + seen1) == sorted(k % 3 for k in range(9))
