"""Launch configurations of the Siddon event kernels and the autotuner.

Every configuration the projector admits (block size, threads per LOR,
ray-length binning of the event order) computes the same operator: forward
projections within 1e-5 relative L2 of the FP64 oracle (and per event within
1e-5 of the one-thread walk), back projections within the 1e-4 image budget,
the adjoint identity to 1e-6.  The autotuner keeps the fastest configuration
it timed and reconstructions with it match the default one.
"""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L

pytestmark = pytest.mark.gpu

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
IP_ARGS = (64, 64, 32, 128, 128, 64)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(tof=None, precision=L.YRTB_COMPENSATED):
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*IP_ARGS)
    pp = yrt.ProjectorParams(sc)
    pp.precision = precision
    if tof:
        pp.addTOF(*tof)
    return sc, ip, yrt.DeviceProjector(sc, ip, pp)


def random_events(n, seed):
    rng = np.random.default_rng(seed)
    osc = po.Scanner(*SC_ARGS)
    d1 = rng.integers(0, osc.num_dets, 3 * n).astype(np.uint32)
    d2 = rng.integers(0, osc.num_dets, 3 * n).astype(np.uint32)
    bins = po.histo3d_bins(osc, d1, d2)
    ok = (bins != np.iinfo(np.uint64).max) & (d1 != d2)
    return d1[ok][:n], d2[ok][:n]


CONFIGS = [(b, t, v) for b in (128, 256) for t in (1, 2, 4)
           for v in (3, 2, 1, 0, 4, 5, 8, 9)
           if not (t > 1 and v != 0)]


@pytest.mark.parametrize("tof", [None, (214.0, 5)])
def test_every_launch_config_vs_oracle(tof):
    sc, ip, p = make(tof)
    d1, d2 = random_events(30000, 41)
    rng = np.random.default_rng(42)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32) if tof else None
    img = rng.random(ip.shape, dtype=np.float32)
    y = rng.random(len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    lors, _ = po.lors_from_detpairs(po.scanner_lut(po.Scanner(*SC_ARGS)), d1, d2)
    oip = po.ImageParams(*IP_ARGS)
    pr = po.Proj(tof_fwhm_ps=tof[0] if tof else 0.0, tof_n_std=tof[1] if tof else 0)
    f64 = po.project(oip, pr, lors, image=img, tof=tv, precision="f64")
    b64 = po.project(oip, pr, lors, values=y.astype(np.float64), tof=tv,
                     forward=False, precision="f64")
    gimg = torch.from_numpy(img).cuda()
    gy = torch.from_numpy(y).cuda()
    base = None
    for block, tpl, vec in CONFIGS:
        p.set_launch(block, tpl, 3, vector_groups=vec)
        assert p.get_launch() == {"block": block, "threads_per_lor": tpl,
                                  "bucket_shift": 3, "order": 0, "tile_shift": 1,
                                  "vector_groups": vec}
        v = p.forward(gimg, ev).cpu().numpy()
        b = p.backward(gy, ev).cpu().numpy()
        # The fused EM pass in every vector mode (float4 gathers, float4 or
        # float2 reductions): the same image up to the FP32 atomics' order.
        em = p.em_step(gimg, torch.zeros(ip.shape, device="cuda"), ev).cpu().numpy()
        if base is None:
            em0 = em
        assert rel_l2(em, em0) < 1e-5, (block, tpl, vec)
        assert rel_l2(v, f64) < 1e-5, (block, tpl)
        assert rel_l2(b, b64) < 1e-4, (block, tpl)
        lhs = float(np.dot(v.astype(np.float64), y))
        rhs = float(np.sum(b.astype(np.float64) * img))
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs), (block, tpl)
        if base is None:
            base = v
        else:
            # Pieces cut at voxel planes: per-event sums differ from the
            # one-thread walk only by rounding.
            d = np.abs(v.astype(np.float64) - base) / np.maximum(np.abs(base), 1e-30)
            assert d.max() < 1e-5, (block, tpl, d.max())


def test_threads_per_lor_needs_compensated_mode():
    sc, ip, p = make((214.0, 5), precision=L.YRTB_MIRROR)
    p.set_launch(128, 1, 2)
    with pytest.raises(yrt.YrtbError, match="threads_per_lor > 1"):
        p.set_launch(256, 2, 3)
    with pytest.raises(yrt.YrtbError, match="block must be"):
        p.set_launch(512, 1, 3)
    with pytest.raises(yrt.YrtbError, match="bucket_shift"):
        p.set_launch(256, 1, 9)
    with pytest.raises(yrt.YrtbError, match="order must be"):
        p.set_launch(256, 1, 3, order=3)
    with pytest.raises(yrt.YrtbError, match="tile_shift"):
        p.set_launch(256, 1, 3, order=1, tile_shift=5)
    with pytest.raises(yrt.YrtbError, match="vector_groups"):
        p.set_launch(256, 1, 3, vector_groups=16)


@pytest.mark.parametrize("shift,order,tile", [(0, 0, 1), (2, 0, 1), (5, 0, 1),
                                              (3, 1, 0), (5, 1, 2), (7, 1, 3),
                                              (4, 2, 1), (7, 2, 0)])
def test_ordering_with_bucket_shift_is_a_subset_major_permutation(shift, order, tile):
    sc, ip, p = make((214.0, 5))
    d1, d2 = random_events(50000, 43)
    tv = np.random.default_rng(44).normal(0, 300, len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    p.set_launch(256, 1, shift, order, tile)
    S = 7
    out, offs = p.order_events(ev, S)
    perm = out.perm.cpu().numpy()
    assert np.array_equal(np.sort(perm), np.arange(len(d1)))
    for s in range(S):
        assert np.all(perm[offs[s]:offs[s + 1]] % S == s)
    # Inside a subset, ray lengths are non-decreasing in buckets of 2^shift
    # of the ordering's O(1) crossing estimate, which exceeds the walk's
    # count by the planes crossed together (ties, a few per ray at most).
    cnt = p.count_crossings(out).cpu().numpy().astype(np.int64)
    for s in range(S):
        c = cnt[offs[s]:offs[s + 1]]
        below = (c[:-1] < (127 << shift) - 8) & (c[1:] < (127 << shift) - 8)
        assert np.all(np.diff(c)[below] >= -(1 << shift) - 4)


def test_autotune_keeps_fastest_and_reconstruction_matches():
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    e = S.generate_events(sc, 60000, 45, tof_fwhm_ps=214.0).numpy()
    outs, reports = [], []
    for tune in (False, True):
        osem = yrt.createOSEM(sc)
        osem.setImageParams(ip)
        osem.num_MLEM_iterations = 2
        osem.num_OSEM_subsets = 3
        osem.setListModeEnabled(True)
        osem.addTOF(214.0, 5)
        osem.projectorParams.precision = L.YRTB_COMPENSATED
        osem.autotune = tune
        osem.generateSensitivityImages()
        lm = yrt.ListModeLUT(sc)
        lm.bind(e["d1"], e["d2"], tof=e["tof"])
        osem.setDataInput(lm)
        outs.append(osem.reconstruct().cpu().numpy())
        reports.append(osem.lastTuneReport)
    rep = reports[1]
    assert 0 < rep["sample_events"] <= (len(e["d1"]) + 2) // 3
    # 3 bucket shifts x 3 orders x 5 vector-group modes, then 2 blocks x
    # 3 threads/LOR minus the stage-1 shape.
    assert len(rep["tried"]) == 3 * 3 * 5 + 2 * 3 - 1
    best_ms = min(ms for _, ms in rep["tried"])
    assert [c for c, ms in rep["tried"] if ms == best_ms][0] == rep["best"]
    assert rel_l2(outs[1], outs[0]) < 1e-5


def test_em_step_same_under_every_order():
    """The EM image of a subset does not depend on the order of its events
    beyond float summation order (image budget 1e-4; here far below)."""
    sc, ip, p = make((214.0, 5))
    d1, d2 = random_events(60000, 47)
    rng = np.random.default_rng(48)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32)
    img = torch.from_numpy(rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)).cuda()
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    S = 3
    ref = None
    for order, tile in [(0, 1), (1, 0), (1, 2), (2, 1)]:
        p.set_launch(256, 1, 3, order, tile)
        out, offs = p.order_events(ev, S)
        em = torch.zeros(ip.shape, device="cuda")
        p.em_step(img, em, out, rng=L.yrtb_range(int(offs[1]), 1, int(offs[2] - offs[1])))
        em = em.cpu().numpy()
        if ref is None:
            ref = em
        else:
            assert rel_l2(em, ref) < 1e-6


def test_release_cached_memory_after_ordering():
    sc, ip, p = make((214.0, 5))
    d1, d2 = random_events(20000, 49)
    tv = np.random.default_rng(50).normal(0, 300, len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    out, offs = p.order_events(ev, 2)
    yrt.release_cached_memory()
    out2, offs2 = p.order_events(ev, 2)   # the pool grows again on demand
    assert torch.equal(out.perm, out2.perm)
