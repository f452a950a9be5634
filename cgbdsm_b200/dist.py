"""Multi-GPU plumbing: one process per GPU (launched by torchrun).

Every rank keeps a full replica of the index and applies every batch; the
matching of a batch is split by seed group: rank r expands the seeds whose
group key (query edge, vertex at the plan's first position) hashes to r
modulo the world size (cgb_config.shard_index / num_shards), so the seeds
of one pendant group stay on one rank.  The batch count is the sum of the
ranks' counts modulo 2^64 (the engine's u64 counter semantics; one
all-reduce per batch, NCCL on GPUs, gloo on CPU), and a step's time is the
maximum over ranks.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env() -> tuple[int, int, int]:
    """(rank, world, local_rank) from the torchrun environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: int = 300) -> None:
    rank, world, local = env()
    if world <= 1 or dist.is_initialized():
        return
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def sum_counts(counts: list[int]) -> list[int]:
    """Element-wise sum over ranks of per-batch match counts, modulo 2^64.

    Counts are u64 values (any value below 2^64, wrapped like the engine's
    own counters).  Each is split into its low and high 32-bit halves, which
    are summed as int64 (exact for up to 2^31 ranks) and recombined."""
    counts = [int(c) % (1 << 64) for c in counts]
    if not dist.is_initialized():
        return counts
    halves = [c & 0xFFFFFFFF for c in counts] + [c >> 32 for c in counts]
    t = torch.tensor(halves, dtype=torch.int64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    s = [int(x) for x in t.tolist()]
    n = len(counts)
    return [(s[i] + (s[n + i] << 32)) % (1 << 64) for i in range(n)]


def max_value(x: float) -> float:
    if not dist.is_initialized():
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def max_values(xs: list[float]) -> list[float]:
    """Element-wise maximum over ranks."""
    if not dist.is_initialized():
        return list(xs)
    t = torch.tensor(xs, dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def barrier() -> None:
    if dist.is_initialized():
        dist.barrier()


def finish() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
