"""Slab sharding across GPUs.

The path shards by 32-slice block with no exchange: a block's reconstruction needs only its own
window of fan views (the reference processes blocks independently, Src/Reconstructor.cpp:33-48).
Rank r of `world` takes a contiguous run of blocks and reads only the fan views those blocks'
windows cover, so no collective is on the data path; the host (or any gather) concatenates the
slabs in rank order.
"""
from __future__ import annotations


def shard_blocks(n_blocks: int, world: int, rank: int, per_rank: int | None = None) -> tuple[int, int]:
    """(first_block, count) of `rank`.  With per_rank, every rank takes that many blocks (weak
    scaling; the scan must plan at least world * per_rank); otherwise the n_blocks are split as
    evenly as possible, earlier ranks taking the remainder."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    if per_rank is not None:
        if per_rank * world > n_blocks:
            raise ValueError(f"{world} x {per_rank} blocks > {n_blocks} planned")
        return rank * per_rank, per_rank
    base, extra = divmod(n_blocks, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def fan_window(plan, first_block: int, count: int) -> tuple[int, int]:
    """[lo, hi) of the fan views blocks [first_block, first_block+count) read."""
    g = plan.info.ctg
    starts = [plan.blocks[b].block_proj_start for b in range(first_block, first_block + count)]
    return min(starts), max(starts) + g.n_angle_add
