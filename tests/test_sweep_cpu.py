"""Replica scheduler (fortress_b200.sweep): balanced partition and the
gather over a world-size-2 gloo group on CPU, with a stand-in for the
per-rank GPU work."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fortress_b200 import sweep


def _insts(k):
    rng = np.random.default_rng(4)
    sizes = rng.choice([128, 192, 256, 384, 512], size=k)
    return [dict(dim=2, spin=1, n=(int(s), int(s)), tag=i) for i, s in enumerate(sizes)]


def test_partition_is_balanced_and_complete():
    insts = _insts(64)
    costs = [sweep.instance_cost(p) for p in insts]
    for world in (1, 2, 3, 8):
        parts, load = sweep.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(insts)))
        assert load == [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(load) <= sum(costs) / world + max(costs)
    assert sweep.partition([5, 5, 5, 5], 2)[0] == [[0, 2], [1, 3]]


def _fake_work(insts, idx):
    return [{"tag": p["tag"], "pts": int(np.prod(p["n"])), "rank": int(os.environ["RANK"])} for p in insts]


def _child(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = sweep.run(_insts(21), _fake_work, rank, world)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.timeout(120)
def test_gather_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_child, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=90) for _ in ps)
    for p in ps:
        p.join(30)
        assert p.exitcode == 0
    insts = _insts(21)
    parts, _ = sweep.partition([sweep.instance_cost(p) for p in insts], 2)
    for r in (0, 1):
        out = res[r]
        assert [o["tag"] for o in out] == list(range(21))          # original order on every rank
        for i, o in enumerate(out):
            assert o["rank"] == (0 if i in parts[0] else 1)
    assert res[0] == res[1]


def test_single_rank_needs_no_group():
    os.environ.setdefault("RANK", "0")
    out = sweep.run(_insts(5), _fake_work)
    assert [o["tag"] for o in out] == list(range(5))
