"""Multi-GPU list-mode OSEM: events sharded across ranks, one exchange per
subset.

Each rank (one process per GPU) holds the full image and its own share of
the events.  A subset's EM-ratio image is the sum of every rank's back
projection, so the ranks all-reduce it (NCCL over NVLink on B200; gloo in
the CPU tests) before applying the same multiplicative update.  No other
data crosses ranks.
"""
from __future__ import annotations

from typing import Callable, Tuple

import torch


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous block [start, stop) of n events owned by rank; blocks differ
    in size by at most one event and cover 0..n-1 exactly once."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("invalid rank / world size")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def subset_of_global_index(global_index, num_subsets: int):
    """OSEM subset of an event (chronological interleaving of the reference,
    BinIteratorChronologicalInterleaved): its global index mod num_subsets."""
    return global_index % num_subsets


def sharded_subset_update(em_local: Callable[[torch.Tensor], None],
                          update: Callable[[torch.Tensor], None],
                          em: torch.Tensor, group=None) -> torch.Tensor:
    """One OSEM subset on a rank: clear em, accumulate this rank's events
    (em_local), sum over ranks, then apply the update with the summed image."""
    em.zero_()
    em_local(em)
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.all_reduce(em, group=group)
    update(em)
    return em
