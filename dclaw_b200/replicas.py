"""Multi-GPU use of the step: independent work per rank, no data-path collective.

A single patch of the benchmark cases fits one B200, and the members of an
ensemble are independent simulations (the reference's particle filters vmap
them; gradient_particle_filter/pf_flume/inference.py:96-108), so several
GPUs run replicas or shards of an ensemble, one process per GPU, and only
the timing is combined: the step time of a run is the maximum over ranks.
"""
from __future__ import annotations

import numpy as np
import torch


def shard_members(cells_per_member, rank: int, world: int) -> list[int]:
    """Member indices of `rank`: contiguous runs of members with about the
    same number of cells per rank (greedy split of the prefix sums)."""
    cells = np.asarray(cells_per_member, dtype=np.float64)
    if world <= 1:
        return list(range(len(cells)))
    bounds = np.cumsum(cells) / cells.sum() * world          # rank boundary positions
    owner = np.minimum((bounds - cells / 2 / cells.sum() * world).astype(int), world - 1)
    return [k for k in range(len(cells)) if owner[k] == rank]


def replica_seed(seed: int, rank: int) -> int:
    """Seed of rank's replica (every rank steps its own synthetic patch)."""
    return seed + rank


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank timing over the ranks of the default group (the
    value itself without one)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
