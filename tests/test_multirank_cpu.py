"""World-size-2 gloo run of the sharded OSEM host logic on CPU.

Each rank owns a contiguous shard of the events, accumulates its EM-ratio
image with the FP64 oracle (standing in for the GPU kernel), and the ranks
all-reduce before the update.  The result must equal the single-process EM
over all events, and the shards must partition the events and preserve each
event's subset (its global index mod the number of subsets).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyyrtpet_b200.distributed import shard_range, sharded_subset_update

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)


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
    ip = po.ImageParams(16, 16, 8, 128, 128, 64)
    img = rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)
    return lors, ip, img


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    sys.path.insert(0, os.path.join(root, "yrt-pet_b200"))
    import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lors, ip, img = _problem()
    n = len(lors)
    subsets, s = 3, 1
    lo, hi = shard_range(n, rank, world)
    gidx = np.arange(lo, hi)
    mine = gidx[gidx % subsets == s]
    em = torch.zeros(ip.shape, dtype=torch.float64)

    def em_local(t):
        t += torch.from_numpy(po.em_step_f64(ip, po.Proj(threads=1), lors[mine], img))

    result = {}

    def update(t):
        result["em"] = t.clone()

    sharded_subset_update(em_local, update, em)
    if rank == 0:
        out.put(result["em"].numpy())
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


def test_two_rank_gloo_em_equals_single_process():
    import pyoracle as po
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    lors, ip, img = _problem()
    n = len(lors)
    full = po.em_step_f64(ip, po.Proj(threads=1), lors[np.arange(1, n, 3)], img)
    np.testing.assert_allclose(got, full, rtol=1e-12, atol=1e-12)
