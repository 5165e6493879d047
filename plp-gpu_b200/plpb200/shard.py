"""Sharding of restarts across ranks (one process per GPU).

Restarts are independent: rank r decodes a contiguous block of the restart
range on its own GPU, with no collective on the data path. Only the final
per-restart summaries (a few dozen bytes each) are gathered, so every rank
can pick the global best with the reference's rule: accepted packings
(score >= theta) first, then the largest (volume, n_boxes), earliest restart
on ties (gpu/plp_common.hpp:493-511, applied across restarts).
"""
from __future__ import annotations


def restart_range(total: int, world: int, rank: int):
    """(first, count) of rank's contiguous block of `total` restarts."""
    if total < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("bad sharding arguments")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def best_restart(summaries):
    """Index of the best summary: (not fallback, volume, n_boxes), earliest on ties.

    summaries: sequence of objects/dicts with fallback, volume, n_boxes."""
    def get(s, k):
        return s[k] if isinstance(s, dict) else getattr(s, k)
    best = None
    for i, s in enumerate(summaries):
        key = (not get(s, "fallback"), get(s, "volume"), get(s, "n_boxes"))
        if best is None or key > best[0]:
            best = (key, i)
    return None if best is None else best[1]


def solve_sharded(solve, total: int, seed: int, group=None):
    """Runs `solve(first_seed, count) -> list of summaries` on this rank's block
    and gathers all ranks' summaries (in restart order) with all_gather_object.
    Returns (summaries of all restarts, index of the global best)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    first, count = restart_range(total, world, rank)
    mine = [dict(volume=s.volume if not isinstance(s, dict) else s["volume"],
                 n_boxes=s.n_boxes if not isinstance(s, dict) else s["n_boxes"],
                 fallback=s.fallback if not isinstance(s, dict) else s["fallback"],
                 score=s.score if not isinstance(s, dict) else s["score"])
            for s in (solve(seed + first, count) if count else [])]
    if world == 1:
        everything = mine
    else:
        parts = [None] * world
        dist.all_gather_object(parts, (first, mine), group=group)
        everything = [s for _, block in sorted(parts, key=lambda p: p[0]) for s in block]
    return everything, best_restart(everything)
