"""Replica / shard plumbing on CPU with the Gloo backend (world size 2):
every unit owned once, max-over-ranks timing, row gather."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "sdf-contact-module_b200"))
    import torch
    import torch.distributed as dist

    from sdfo.distributed import gather_rows, max_over_ranks, shard_range

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 1001
        a, b = shard_range(n, rank, world)
        t = max_over_ranks(10.0 + rank)
        local = torch.arange(a, b, dtype=torch.float64).reshape(-1, 1).repeat(1, 6)
        full = gather_rows(local, n)
        q.put((rank, a, b, t, full[:, 0].tolist()))
    finally:
        dist.destroy_process_group()


def test_shard_range_partitions():
    from sdfo.distributed import shard_range

    for n in (0, 1, 7, 1000, 4096):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_two_rank_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    import queue
    import time

    res = []
    deadline = time.time() + 120
    while len(res) < 2 and time.time() < deadline:
        try:
            res.append(q.get(timeout=1))
        except queue.Empty:
            if any(p.exitcode not in (None, 0) for p in procs):
                break
    for p in procs:
        p.join(timeout=60)
        if p.exitcode is None:
            p.kill()
        assert p.exitcode == 0
    assert len(res) == 2
    res.sort()
    assert res[0][1:3] == (0, 501) and res[1][1:3] == (501, 1001)
    assert all(r[3] == 11.0 for r in res)
    assert all(r[4] == list(range(1001)) for r in res)
