"""Multi-rank plumbing on CPU (gloo, world size 2): shard counts are summed and
step times reduced by max, as bench.py does over NCCL on GPUs."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from cgbdsm_b200 import dist

    dist.init("gloo", timeout_s=60)
    counts = dist.sum_counts([10 * rank + 1, 2**40 + rank, 0])
    t = dist.max_value(1.5 + rank)
    dist.barrier()
    dist.finish()
    q.put((rank, counts, t))


def test_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, counts, t in out:
        assert counts == [1 + 11, 2**41 + 1, 0]
        assert t == 2.5


def test_single_process_is_identity():
    from cgbdsm_b200 import dist

    assert dist.sum_counts([3, 4]) == [3, 4]
    assert dist.max_value(1.25) == 1.25
