"""Multi-rank plumbing on CPU (gloo, world size 2): shard counts are summed
modulo 2^64 and step times reduced by max, as bench.py does over NCCL on GPUs.

The shard counts are real ones: each rank runs the oracle's per-edge count
restricted to its shard of the seed groups (the engine's shard key: query
edge and the data vertex at the plan's first position, hashed) on the same
batch stream, and the all-reduced sums must equal the unsharded counts."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_counts(rank, world, workdir):
    """Per-batch counts of one shard (world > 1) or of all seeds, on t_er5."""
    from cgbdsm_b200 import Producer
    from cgbdsm_b200.workloads import SPECS, materialize, read_query
    from oracle import bind

    spec = SPECS["t_er5"]
    p = materialize(spec, workdir)
    ql, qe = read_query(p["query"])
    prod = Producer(p["query"], p["data"], p["update"], spec.cli_batch_size, threads=1)
    init, dv = prod.initial()
    orc = bind.Oracle(len(ql), qe)
    if world > 1:
        orc.set_shard(rank, world)
    orc.build(init, dv)
    out = []
    for _ in range(prod.num_batches):
        r = prod.next()
        out.append(orc.batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"], bind.PER_EDGE))
    prod.close()
    return out


def _worker(rank, world, port, workdir, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from cgbdsm_b200 import dist

    dist.init("gloo", timeout_s=120)
    counts = dist.sum_counts([10 * rank + 1, 2**40 + rank, 0])
    # u64 counts: sums wrap modulo 2^64 like the engine's counters
    wide = dist.sum_counts([2**63 + 5 + 2 * rank, 2**64 - 1 if rank == 0 else 1, 2**63 + rank])
    t = dist.max_value(1.5 + rank)
    mine = _shard_counts(rank, world, workdir)
    shard_sum = dist.sum_counts(mine)
    dist.barrier()
    dist.finish()
    q.put((rank, counts, wide, t, mine, shard_sum))


def test_gloo_two_ranks(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=300) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = _shard_counts(0, 1, str(tmp_path))
    assert sum(full) > 0
    for rank, counts, wide, t, mine, shard_sum in out:
        assert counts == [1 + 11, 2**41 + 1, 0]
        assert wide == [12, 0, 1]
        assert t == 2.5
        assert shard_sum == full, "shard counts do not add up to the unsharded counts"
    # both shards hold seeds
    assert all(sum(o[4]) > 0 for o in out)


def test_single_process_is_identity():
    from cgbdsm_b200 import dist

    assert dist.sum_counts([3, 4]) == [3, 4]
    assert dist.sum_counts([2**64 + 3]) == [3]
    assert dist.max_value(1.25) == 1.25
