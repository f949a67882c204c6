"""Multi-GPU list-mode OSEM: events sharded across ranks, one exchange per
subset.

Each rank (one process per GPU) holds the full image and its own contiguous
share of the events.  An event keeps the subset the reference gives it in
the whole stream, its global index mod the number of subsets
(BinIteratorChronologicalInterleaved, src/datastruct/projection/
BinIterator.cpp:261-265), wherever the shard boundaries fall.  A subset's
EM-ratio image is the sum of every rank's back projection, so the ranks
all-reduce it (NCCL over NVLink on B200; gloo in the CPU tests) before
applying the same multiplicative update.  The sensitivity image is split the
same way: each rank back-projects its share of the histogram's parts and one
all-reduce sums them.  No other data crosses ranks.

The loop itself (osem_loop) takes the EM pass and the update as callables,
so that the host logic runs unchanged over the C ABI on GPUs and over a CPU
stand-in in the tests.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np
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


def local_subset_range(n_local: int, first_global_index: int,
                       num_subsets: int, subset: int) -> Tuple[int, int, int]:
    """(start, stride, count) of the local events of one subset in a shard of
    n_local events whose first event has global index first_global_index:
    the local events e with (first_global_index + e) mod num_subsets ==
    subset, in file order (the yrtb_range of an unordered shard)."""
    k = (subset - first_global_index) % num_subsets
    count = 0 if n_local <= k else (n_local - k + num_subsets - 1) // num_subsets
    return k, num_subsets, count


def local_subset_indices(n_local: int, first_global_index: int,
                         num_subsets: int, subset: int) -> np.ndarray:
    start, stride, count = local_subset_range(n_local, first_global_index,
                                              num_subsets, subset)
    return start + stride * np.arange(count, dtype=np.int64)


def subset_ranges(n_local: int, num_subsets: int, first_global_index: int = 0,
                  offsets: Optional[Sequence[int]] = None):
    """The (start, stride, count) of every subset of a shard: contiguous
    blocks when the shard was ordered subset-major (offsets from
    DeviceProjector.order_events(..., first_global_index)), else the
    interleaved ranges of local_subset_range."""
    if offsets is not None:
        return [(int(offsets[s]), 1, int(offsets[s + 1] - offsets[s]))
                for s in range(num_subsets)]
    return [local_subset_range(n_local, first_global_index, num_subsets, s)
            for s in range(num_subsets)]


def _all_reduce(t: torch.Tensor, group=None):
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.all_reduce(t, group=group)


def sharded_subset_update(em_local: Callable[[torch.Tensor], None],
                          update: Callable[[torch.Tensor], None],
                          em: torch.Tensor, group=None) -> torch.Tensor:
    """One OSEM subset on a rank: clear em, accumulate this rank's events
    (em_local), sum over ranks, then apply the update with the summed image."""
    em.zero_()
    em_local(em)
    _all_reduce(em, group)
    update(em)
    return em


def osem_loop(iterations: int, num_subsets: int, em: torch.Tensor,
              em_pass: Callable[[int, torch.Tensor], None],
              update: Callable[[torch.Tensor], None], group=None):
    """The OSEM subset loop of one rank (OSEM::reconstruct, src/recon/
    OSEM.cpp:315-365): for every iteration and subset s, em_pass(s, em) adds
    this rank's back projection of subset s into em, the ranks sum em, and
    update(em) applies the multiplicative update.  Every rank takes the same
    collective steps in the same order."""
    for _ in range(iterations):
        for s in range(num_subsets):
            sharded_subset_update(lambda buf, s=s: em_pass(s, buf), update, em,
                                  group=group)


def sensitivity_parts(num_parts: int, rank: int, world: int) -> list:
    """The histogram parts (phi-interleaved subsets of the bins) one rank
    back-projects for the sensitivity image: parts rank, rank+world, ..."""
    return list(range(rank, num_parts, world))


def sensitivity_histo3d(proj, sens: torch.Tensor, num_parts: int = 20,
                        group=None, **kw) -> torch.Tensor:
    """Sensitivity image over all histogram bins, split across the ranks:
    each rank back-projects its parts (DeviceProjector.sensitivity_histo3d,
    kw: mu, mu_params, crystal_eff, sens_histo, acf_histo), then one
    all-reduce sums them (before the hard threshold, which the caller
    applies)."""
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        rank = torch.distributed.get_rank(group)
        world = torch.distributed.get_world_size(group)
    else:
        rank, world = 0, 1
    for part in sensitivity_parts(num_parts, rank, world):
        proj.sensitivity_histo3d(sens, num_parts, part, **kw)
    _all_reduce(sens, group)
    return sens


def osem_listmode(proj, events, offsets, sens: torch.Tensor, img: torch.Tensor,
                  iterations: int, subsets: int, global_scale: float = 1.0,
                  denom_threshold: float = 1e-35, init_from_image: bool = False,
                  group=None, first_global_index: int = 0) -> torch.Tensor:
    """List-mode OSEM over this rank's shard of the events, with the EM-ratio
    image summed over ranks once per subset.  offsets: the subset offsets of
    DeviceProjector.order_events(events, subsets, first_global_index) for a
    subset-major shard, or None for events in file order (then the shard's
    first event has global index first_global_index).  Same steps as
    yrtb_osem_listmode (x0 = 0.125 masked by sens > 0, sensitivity /
    subsets, EM update with threshold EPS_FLT), driven from Python so that
    the collective sits between the EM pass and the update."""
    import ctypes
    from . import _lib as L
    from .core import _stream
    lib = L.lib()
    ip = proj.img_params
    J, nt = ip.numVoxels, ip.nt
    em = torch.empty(nt * J, dtype=torch.float32, device=img.device)
    sens_sub = (sens.reshape(-1)[:J] / float(subsets)).contiguous()
    s_ptr = _stream()
    if not init_from_image:
        L.check(lib.yrtb_fill(img.data_ptr(), nt * J, 0.125, s_ptr))
    L.check(lib.yrtb_apply_threshold(img.data_ptr(), sens.data_ptr(), J, nt, 1,
                                     0.0, 0.0, 0.0, 1.0, 0.0, s_ptr))
    evc = events.c()
    ranges = subset_ranges(events.count, subsets, first_global_index, offsets)

    def em_pass(s, buf):
        start, stride, count = ranges[s]
        if count:
            L.check(lib.yrtb_em_step(proj.h, img.data_ptr(), buf.data_ptr(),
                                     ctypes.byref(evc),
                                     L.yrtb_range(start, stride, count),
                                     float(global_scale), float(denom_threshold),
                                     s_ptr))

    def update(buf):
        L.check(lib.yrtb_em_update(img.data_ptr(), buf.data_ptr(), sens_sub.data_ptr(),
                                   J, nt, 1, 1.19209e-07, None, s_ptr))

    osem_loop(iterations, subsets, em, em_pass, update, group=group)
    return img
