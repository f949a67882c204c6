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


def osem_listmode(proj, events, offsets, sens: torch.Tensor, img: torch.Tensor,
                  iterations: int, subsets: int, global_scale: float = 1.0,
                  denom_threshold: float = 1e-35, init_from_image: bool = False,
                  group=None) -> torch.Tensor:
    """List-mode OSEM over this rank's share of the events (already in
    subset-major order, subset s = events [offsets[s], offsets[s+1])), with
    the EM-ratio image summed over ranks once per subset.  Same steps as
    yrtb_osem_listmode (x0 = 0.125 masked by sens > 0, sensitivity / subsets,
    EM update with threshold EPS_FLT), driven from Python so that the
    collective sits between the EM pass and the update."""
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

    def em_local(s):
        def run(buf):
            r = L.yrtb_range(int(offsets[s]), 1, int(offsets[s + 1] - offsets[s]))
            if r.count:
                L.check(lib.yrtb_em_step(proj.h, img.data_ptr(), buf.data_ptr(),
                                         ctypes.byref(evc), r, float(global_scale),
                                         float(denom_threshold), s_ptr))
        return run

    def update(buf):
        L.check(lib.yrtb_em_update(img.data_ptr(), buf.data_ptr(), sens_sub.data_ptr(),
                                   J, nt, 1, 1.19209e-07, None, s_ptr))

    for _ in range(iterations):
        for s in range(subsets):
            sharded_subset_update(em_local(s), update, em, group=group)
    return img
