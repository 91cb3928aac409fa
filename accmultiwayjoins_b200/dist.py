"""Multi-GPU plumbing for the join operators (one process per GPU).

The join path shards without a data-path exchange: the probe relation's rows
split into contiguous ranges, one per rank, joined against the other
relations whole (replicated build indexes).  Every result tuple extends
exactly one probe row, so the ranks' results partition the query's.  The
only exchange is the final 16-byte (count, checksum) sum, done here with
torch.distributed (NCCL on GPUs, gloo on CPU).  Both values add modulo 2^64:
they travel as int64, whose addition wraps the same way.
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


def shard_relation(relation, rank: int, world: int):
    """Rank `rank`'s share of a (columns, attrs) relation: rows [lo, hi)."""
    cols, attrs = relation
    lo, hi = shard_range(len(cols[0]), rank, world)
    return [c[lo:hi] for c in cols], attrs


def sharded_join(ctx, relations, rank: int, world: int, op: str = "amhj", reduce: bool = True, group=None,
                 device=None, **kw):
    """One NORMAL query over `world` ranks.  relations: (columns, attrs)
    pairs, the first the probe relation; this rank joins its share of the
    probe rows with the others whole, through ctx.amhj (op "amhj": the
    first relation is the probe) or ctx.lftj (op "lftj": the first
    relation's share is the first trie; relations without repeated rows, as
    the leapfrog triejoin joins sets).  With reduce, the (count, checksum) pairs are summed over
    the process group; otherwise this rank's pair is returned.  A triangle or
    4-clique over one edge relation is sharded as its NORMAL form: the edge
    relation once per attribute pair, e.g. (0,1), (1,2), (0,2)."""
    mine = [shard_relation(relations[0], rank, world)] + list(relations[1:])
    handles = [ctx.relation(c, a) for c, a in mine]
    try:
        if op == "amhj":
            r = ctx.amhj("NORMAL", handles, **kw)
        elif op == "lftj":
            r = ctx.lftj(handles, **kw)
        else:
            raise ValueError("op must be amhj or lftj")
    finally:
        for h in handles:
            h.release()
    if not reduce or world == 1:
        return r.count, r.checksum
    return allreduce_result(r.count, r.checksum, device=device, group=group)
