"""Frequency partition + result gather across 2 ranks (gloo on CPU, world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from emerge_b200 import distributed


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, systems, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = distributed.run_partitioned(systems, lambda batch: [(f * 2.0, p, rank) for f, p in batch],
                                          world, rank, batch=3)
        out_q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_system_once():
    systems = [(float(f), p) for f in range(11) for p in range(2)]
    shares = [distributed.partition(systems, 3, r) for r in range(3)]
    idx = sorted(i for s in shares for i, _ in s)
    assert idx == list(range(len(systems)))
    with pytest.raises(ValueError):
        distributed.partition(systems, 2, 2)


def test_gather_detects_missing():
    with pytest.raises(RuntimeError):
        distributed.gather([(0, "a")], 2)


def test_two_rank_gloo_sweep_partition():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    systems = [(float(f), p) for f in range(7) for p in range(2)]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, systems, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, res in results:
        assert len(res) == len(systems)
        for i, (v, port_, solver_rank) in enumerate(res):
            assert v == systems[i][0] * 2.0 and port_ == systems[i][1]
            assert solver_rank == i % 2       # round-robin ownership
