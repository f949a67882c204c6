"""Benchmark-size workloads, checked through properties that hold at any size.

At the benchmark configurations' own sizes the oracle cannot check every
output, so these tests check what does not depend on size: agreement with
the FP64 oracle on a seeded sample of the events, the adjoint identity over
all events, linearity of the EM back projection over event subsets, the
per-event invariance of projections under the device event ordering, and the
exact count checksum of list-mode binning.

Tolerances: forward projections 1e-5 relative L2 against FP64; images 1e-6
where the same FP32 terms are only summed in another order; adjoint 1e-6;
binning exact.
"""
import ctypes

import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L
from pyyrtpet_b200 import synthetic as S

pytestmark = pytest.mark.gpu

# 80 rings x 672 crystals, radius 410 mm, 3.2 mm pitch (the TOF list-mode
# benchmark scanner) and its 256 x 256 x 160 image at 2 mm.
C2 = (256, 3.2, 3.2, 20, 410, 672, 80, 1, 79, 2, 1)
C2_IMAGE = (256, 256, 160, 512, 512, 320)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def c2():
    sc = S.scanner_c2()
    ip = S.image_c2()
    assert (ip.nx, ip.ny, ip.nz) == C2_IMAGE[:3]
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = L.YRTB_COMPENSATED
    p = yrt.DeviceProjector(sc, ip, pp)
    evs = S.generate_events(sc, 4_000_000, 20261203 + 101, tof_fwhm_ps=214.0,
                            randoms_fraction=0.2, device="cuda", chunk=1 << 23)
    ev = yrt.DeviceEvents(int(evs.d1.numel()), evs.d1.to(torch.int32).contiguous(),
                          evs.d2.to(torch.int32).contiguous(), tof=evs.tof.contiguous())
    g = torch.Generator(device="cuda")
    g.manual_seed(102)
    img = (0.5 + torch.rand(ip.shape, generator=g, device="cuda")).contiguous()
    return sc, ip, p, ev, img


def test_c2_forward_sample_vs_fp64_and_adjoint(c2):
    sc, ip, p, ev, img = c2
    fwd = p.forward(img, ev)
    # A seeded sample of 20k events against the FP64 oracle.
    rng = np.random.default_rng(103)
    idx = np.sort(rng.choice(ev.count, 20000, replace=False))
    d1 = ev.d1.cpu().numpy().view(np.uint32)[idx]
    d2 = ev.d2.cpu().numpy().view(np.uint32)[idx]
    tof = ev.tof.cpu().numpy()[idx]
    lors, _ = po.lors_from_detpairs(po.scanner_lut(po.Scanner(*C2)), d1, d2)
    ref = po.project(po.ImageParams(*C2_IMAGE), po.Proj(tof_fwhm_ps=214.0, tof_n_std=5),
                     lors, image=img.cpu().numpy(), tof=tof, precision="f64")
    assert rel_l2(fwd.cpu().numpy()[idx], ref) < 1e-5
    # Adjoint identity <A x, y> = <x, A^T y> over all 4M events.
    g = torch.Generator(device="cuda")
    g.manual_seed(104)
    y = torch.rand(ev.count, generator=g, device="cuda")
    b = p.backward(y, ev)
    lhs = float(torch.dot(fwd.double(), y.double()))
    rhs = float(torch.sum(b.double() * img.double()))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def test_c2_ordering_keeps_projections_and_em_is_linear_over_subsets(c2):
    sc, ip, p, ev, img = c2
    fwd = p.forward(img, ev)
    ordered, offs = p.order_events(ev, 10)
    # Every event keeps its own projection, bit for bit, in the new order.
    fwd_o = p.forward(img, ordered)
    assert torch.equal(fwd_o, fwd[ordered.perm])
    # The EM back projection is linear in the events: the 10 subsets summed
    # into one image equal one pass over all events (FP32 sums reordered).
    em_all = torch.zeros(ip.shape, device="cuda")
    p.em_step(img, em_all, ordered)
    em_sub = torch.zeros(ip.shape, device="cuda")
    for s in range(10):
        a, b = int(offs[s]), int(offs[s + 1])
        p.em_step(img, em_sub, ordered, rng=L.yrtb_range(a, 1, b - a))
    assert rel_l2(em_sub.cpu().numpy(), em_all.cpu().numpy()) < 1e-6
    # And the same pass over the events in file order.
    em_file = torch.zeros(ip.shape, device="cuda")
    p.em_step(img, em_file, ev)
    assert rel_l2(em_file.cpu().numpy(), em_all.cpu().numpy()) < 1e-6


def test_c3_binning_count_checksum_50m_events():
    # The histogram benchmark's scanner (16 rings x 256, all ring differences)
    # and 50M events, a quarter of its 200M: plus 2 % raw detector pairs,
    # some of them d1 == d2, which the binning must skip.
    sc = S.scanner_c1(15)
    p = yrt.core._scratch_projector(sc)
    h = yrt.Histogram3D(sc)
    n = 50_000_000
    evs = S.generate_events(sc, n - n // 50, 20261203 + 105, device="cuda", chunk=1 << 24)
    g = torch.Generator(device="cuda")
    g.manual_seed(106)
    raw = torch.randint(0, sc.getNumDets(), (2, n // 50), generator=g, device="cuda",
                        dtype=torch.int32)
    raw[1, ::17] = raw[0, ::17]
    d1 = torch.cat([evs.d1.to(torch.int32), raw[0]]).contiguous()
    d2 = torch.cat([evs.d2.to(torch.int32), raw[1]]).contiguous()
    del evs
    hist = torch.zeros(h.histoSize, dtype=torch.float32, device="cuda")
    bad = ctypes.c_uint64()
    # Pairs outside the histogram (minimum angle difference) are counted and
    # reported with YRTB_ERR_RANGE; the valid ones are binned all the same.
    status = L.lib().yrtb_listmode_to_histo3d(p.h, d1.data_ptr(), d2.data_ptr(), None,
                                              d1.numel(), hist.data_ptr(),
                                              ctypes.byref(bad), None)
    assert bad.value > 0 and status == L.YRTB_ERR_RANGE
    bins = torch.empty(d1.numel(), dtype=torch.int64, device="cuda")
    L.check(L.lib().yrtb_histo3d_bins(p.h, d1.data_ptr(), d2.data_ptr(), d1.numel(),
                                      bins.data_ptr(), None))
    valid = (bins != -1) & (d1 != d2)
    nvalid = int(valid.sum())
    # Counts are exact integers in FP32 (every bin < 2^24): the histogram sums
    # to the number of binned events, and equals the per-bin count of the
    # bin indices that the separate map kernel gives.
    assert float(hist.double().sum()) == float(nvalid)
    assert nvalid + int(bad.value) + int((d1 == d2).sum()) == d1.numel()
    counts = torch.bincount(bins[valid], minlength=h.histoSize).float()
    assert torch.equal(counts, hist)
    # The bin map itself against the oracle on the 1M raw pairs.
    a = d1[-1_000_000:].cpu().numpy().view(np.uint32)
    b = d2[-1_000_000:].cpu().numpy().view(np.uint32)
    ok = a != b
    a, b = a[ok], b[ok]
    ref = po.histo3d_bins(po.Scanner(64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1), a, b)
    assert np.array_equal(yrt.histo3d_bins(sc, a, b), ref)
