"""World-size-2 gloo runs of the sharded OSEM host logic on CPU.

The ranks run pyyrtpet_b200.distributed's own loop (osem_loop, the subset
ranges of a shard, the all-reduce per subset); the EM pass of a rank is the
FP64 oracle over the rank's events of the subset (standing in for the GPU
kernel, which needs a GPU).  Shards are contiguous blocks whose starts are
not multiples of the number of subsets, so every event must keep its
subset of the whole stream (global index mod subsets,
BinIteratorChronologicalInterleaved, src/datastruct/projection/
BinIterator.cpp:261-265).  The reconstructed image must equal one process
running the same loop over all events (rtol 1e-6: the EM pass reads the
image in FP32, so a last-bit difference of the FP64 sums may round one voxel
the other way; a wrong subset would differ by percents), with the shard in
file order and in subset-major order (the offsets DeviceProjector.
order_events returns).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyyrtpet_b200.distributed import (local_subset_indices, local_subset_range,
                                       osem_loop, sensitivity_parts, shard_range,
                                       subset_ranges, sharded_subset_update)

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
SUBSETS = 7
ITERATIONS = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _problem():
    import pyoracle as po
    rng = np.random.default_rng(71)
    sc = po.Scanner(*SC_ARGS)
    d1 = rng.integers(0, sc.num_dets, 9000)
    d2 = rng.integers(0, sc.num_dets, 9000)
    ok = (d1 % 256) != (d2 % 256)
    lors, _ = po.lors_from_detpairs(po.scanner_lut(sc), d1[ok], d2[ok])
    lors = lors[:8957]   # two shards of 4479 and 4478: rank 1 starts at 4479 = 6 mod 7
    ip = po.ImageParams(16, 16, 8, 128, 128, 64)
    sens = rng.uniform(50.0, 150.0, ip.shape)
    return lors, ip, sens


def _reconstruct(lors_local, first, ip, sens, ordered, group=None):
    """The sharded loop of distributed.osem_loop with an FP64 CPU EM pass."""
    import pyoracle as po
    n = len(lors_local)
    offsets = None
    if ordered:
        # Subset-major order of the shard (what order_events produces).
        key = (first + np.arange(n)) % SUBSETS
        perm = np.argsort(key, kind="stable")
        lors_local = lors_local[perm]
        offsets = np.concatenate([[0], np.cumsum(np.bincount(key, minlength=SUBSETS))])
    ranges = subset_ranges(n, SUBSETS, first, offsets)
    x = torch.full(ip.shape, 0.125, dtype=torch.float64)
    sens_sub = torch.from_numpy(sens) / SUBSETS
    em = torch.zeros(ip.shape, dtype=torch.float64)

    def em_pass(s, buf):
        start, stride, count = ranges[s]
        sel = start + stride * np.arange(count)
        if count:
            buf += torch.from_numpy(po.em_step_f64(
                ip, po.Proj(threads=1), lors_local[sel], x.float().numpy()))

    def update(buf):
        x.mul_(torch.where(sens_sub > 1.19209e-07, buf / sens_sub,
                           torch.ones_like(buf)))

    osem_loop(ITERATIONS, SUBSETS, em, em_pass, update, group=group)
    return x.numpy()


def _worker(rank, world, port, ordered, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    sys.path.insert(0, os.path.join(root, "yrt-pet_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lors, ip, sens = _problem()
    lo, hi = shard_range(len(lors), rank, world)
    img = _reconstruct(lors[lo:hi], lo, ip, sens, ordered)
    if rank == 0:
        out.put((lo, hi, img))
    else:
        out.put((lo, hi, None))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range_partitions():
    for n in (0, 1, 7, 100, 101):
        for w in (1, 2, 3, 8):
            cover = []
            for r in range(w):
                a, b = shard_range(n, r, w)
                cover.extend(range(a, b))
                assert b - a in (n // w, n // w + 1)
            assert cover == list(range(n))


def test_local_subset_ranges_keep_global_subsets():
    # Shards cut anywhere: local event e of a shard starting at `first`
    # belongs to subset (first + e) mod S, and the subsets of all shards
    # together are exactly the interleaved subsets of the whole stream.
    for n, S in ((100, 7), (101, 3), (64, 64), (5, 9)):
        for world in (1, 2, 3, 4):
            for s in range(S):
                got = []
                for r in range(world):
                    lo, hi = shard_range(n, r, world)
                    idx = local_subset_indices(hi - lo, lo, S, s)
                    assert np.all((lo + idx) % S == s)
                    start, stride, count = local_subset_range(hi - lo, lo, S, s)
                    assert count == len(idx) and stride == S
                    got.extend((lo + idx).tolist())
                assert sorted(got) == list(range(s, n, S))


def test_sensitivity_parts_partition():
    for parts in (1, 7, 20):
        for world in (1, 2, 3, 8):
            cover = sorted(p for r in range(world)
                           for p in sensitivity_parts(parts, r, world))
            assert cover == list(range(parts))


@pytest.mark.parametrize("ordered", [False, True])
def test_two_rank_gloo_osem_equals_single_process(ordered):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ordered, q))
             for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    lors, ip, sens = _problem()
    starts = sorted(r[0] for r in results)
    assert any(s % SUBSETS for s in starts)   # a shard boundary inside a stride
    got = next(r[2] for r in results if r[2] is not None)
    full = _reconstruct(lors, 0, ip, sens, ordered=False)
    np.testing.assert_allclose(got, full, rtol=1e-6, atol=1e-12)


def test_sharded_subset_update_single_process():
    em = torch.ones(4, dtype=torch.float64)
    seen = {}
    sharded_subset_update(lambda t: t.add_(2.0), lambda t: seen.setdefault("em", t.clone()), em)
    assert torch.equal(seen["em"], torch.full((4,), 2.0, dtype=torch.float64))
