"""One graph counted on several GPUs: one process per GPU, each holding the
whole oriented graph and counting one unit shard (kc_count_shard), then one
exact sum of the shards' 128-bit counts over torch.distributed.

The units (node or edge units, as kc_count's) are dealt out by position
inside their size class, so every shard gets a share of every size and the
few largest units of a power-law graph land on different GPUs. The only data
exchanged is the count: 16 bytes per rank, as four 32-bit limbs in int64
lanes, all-reduced with SUM (exact for up to 2^31 ranks) and carried on the
host. No reference counterpart: the reference counts one graph on one GPU
(its unit windows, kclique/kclique.cuh:1645-1675, run one after another).
"""
from __future__ import annotations

LIMBS = 4  # 32-bit limbs of an unsigned 128-bit count


def to_limbs(value: int) -> list[int]:
    if value < 0 or value >> 128:
        raise ValueError("count outside the unsigned 128-bit range")
    return [(value >> (32 * i)) & 0xFFFFFFFF for i in range(LIMBS)]


def from_limb_sums(sums) -> int:
    """The 128-bit total from per-limb sums (each below 2^63): carries move up."""
    total = 0
    for i, s in enumerate(sums):
        total += int(s) << (32 * i)
    if total >> 128:
        raise OverflowError("the shards' counts add up to more than 128 bits")
    return total


def sum_u128(value: int, pg=None) -> int:
    """Exact sum of a non-negative 128-bit integer over the ranks of the
    process group (default group when pg is None). NCCL groups reduce on the
    current CUDA device, others (gloo) on the host."""
    import torch
    import torch.distributed as dist

    device = "cpu"
    if dist.get_backend(pg) == "nccl":
        device = f"cuda:{torch.cuda.current_device()}"
    t = torch.tensor(to_limbs(value), dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=pg)
    return from_limb_sums(t.cpu().tolist())


def count_shard(graph, k: int, rank: int, world: int, **params):
    """This rank's shard of graph.count(k, **params) (kc_count_shard)."""
    return graph.count(k, shard=(rank, world), **params)


def count_sharded(graph, k: int, pg=None, **params) -> int:
    """graph.count(k, **params) split over the ranks of the process group:
    every rank passes its own copy of the same oriented graph and gets the
    whole count back."""
    import torch.distributed as dist

    rank, world = dist.get_rank(pg), dist.get_world_size(pg)
    mine = count_shard(graph, k, rank, world, **params)
    if params.get("stats"):
        mine = mine.count
    return sum_u128(int(mine), pg)
