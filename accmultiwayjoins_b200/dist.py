"""Multi-GPU plumbing for the join operators (one process per GPU).

The join path shards without a data-path exchange: probe rows (AMHJ) or the
level-1 entries of the first trie (ALFTJ) split into contiguous ranges, one
per rank, against replicated build indexes.  The only exchange is the final
16-byte (count, checksum) sum, done here with torch.distributed (NCCL on
GPUs, gloo on CPU).  Both values add modulo 2^64: they travel as int64,
whose addition wraps the same way.
"""
from __future__ import annotations

M64 = (1 << 64) - 1


def shard_range(n: int, rank: int, world: int):
    """Contiguous share [lo, hi) of n units for `rank` of `world`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    return n * rank // world, n * (rank + 1) // world


def _to_i64(v: int) -> int:
    v &= M64
    return v - (1 << 64) if v >= (1 << 63) else v


def allreduce_result(count: int, checksum: int, device=None, group=None):
    """Sum (count, checksum) over the ranks of the process group, mod 2^64."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([_to_i64(count), _to_i64(checksum)], dtype=torch.int64, device=device)
    dist.all_reduce(t, group=group)
    return int(t[0].item()) & M64, int(t[1].item()) & M64
