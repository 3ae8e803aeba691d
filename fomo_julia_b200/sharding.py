"""Shots over several GPUs: one process per GPU, shots sharded by rank.

Shots are independent (no exchange during time stepping), so the multi-GPU
form of ``run_shots!`` (src/simulation/shot_manager.jl:145-180) gives each
rank every world-th shot, runs them on its own GPU (single shots or one batch)
and gathers the seismograms to rank 0 at the end -- the only collective.
``torch.distributed`` carries the gather (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np


def shard(n_shots: int, world: int, rank: int) -> List[int]:
    """Shot indices of `rank`: rank, rank + world, ... (round robin, so ranks
    differ by at most one shot)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    if n_shots < 0:
        raise ValueError(f"n_shots={n_shots} < 0")
    return list(range(rank, n_shots, world))


def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return None
    return dist


def max_over_ranks(value: float) -> float:
    """Largest value over the ranks (the job's time is its slowest rank's)."""
    dist = _dist()
    if dist is None:
        return float(value)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, float(value))
    return max(out)


def run_sharded(run: Callable[[Sequence[int]], List[object]], n_shots: int) -> Optional[List[object]]:
    """Runs this rank's shots with `run(indices) -> results` (one result per
    index, in order) and gathers every rank's results to rank 0, which gets
    the n_shots results in shot order; the other ranks get None.  Without an
    initialised process group the whole job is one rank."""
    dist = _dist()
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    mine = shard(n_shots, world, rank)
    res = run(mine)
    if len(res) != len(mine):
        raise RuntimeError(f"rank {rank}: {len(res)} results for {len(mine)} shots")
    if dist is None:
        return list(res)
    parts = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, res)), parts, dst=0)
    if rank != 0:
        return None
    out: List[object] = [None] * n_shots
    for part in parts:
        for k, r in part:
            out[k] = r
    return out


def run_shots_distributed(b, W, M, H, a, rec_template, shot_config, params, batched: bool = True):
    """run_shots! over all ranks: each rank runs its shard of
    `shot_config.shots` on its GPU (one batch, or one shot after another with
    batched=False) and rank 0 returns every ShotResult in shot order."""
    from . import elastic2d as E

    def run(idx):
        cfg = E.MultiShotConfig([shot_config.shots[k] for k in idx], shot_config.wavelet, shot_config.source_type)
        if not idx:
            return []
        return E.run_shots(b, W, M, H, a, rec_template, cfg, params, batched=batched)

    return run_sharded(run, len(shot_config.shots))


def gathers_equal(a: List[np.ndarray], b: List[np.ndarray]) -> bool:
    return len(a) == len(b) and all(np.array_equal(x, y) for x, y in zip(a, b))
