"""CUDA path (through the C ABI) against the reference and the oracle.

Tolerances (stated per test): bit-exact for integer work (detector LUT,
histogram maps, list-mode binning) and for non-TOF forward projections in
mirror mode; relative L2 <= 1e-5 per projection vector and <= 1e-4 per image
against the FP64 oracle or the reference; adjoint identity to 1e-6.
"""
import os

import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "ref_small.npz"))
SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
IP_ARGS = (32, 32, 16, 128, 128, 64)
needs_ref = pytest.mark.skipif(not po.ref_available(),
                               reason="reference library not built")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def make(sc_args=SC_ARGS, ip_args=IP_ARGS, projector="S", tof=None,
         num_rays=1, psf=None, precision=L.YRTB_MIRROR, nt=1):
    sc = yrt.Scanner("t", *sc_args)
    ip = yrt.ImageParams(*ip_args, nt=nt)
    pp = yrt.ProjectorParams(sc)
    pp.setProjector(projector)
    pp.numRays = num_rays
    pp.precision = precision
    if tof:
        pp.addTOF(*tof)
    if psf is not None:
        pp.setProjPsf(*psf)
    return sc, ip, yrt.DeviceProjector(sc, ip, pp)


def random_events(sc_args, n, seed):
    rng = np.random.default_rng(seed)
    osc = po.Scanner(*sc_args)
    d1 = rng.integers(0, osc.num_dets, 3 * n).astype(np.uint32)
    d2 = rng.integers(0, osc.num_dets, 3 * n).astype(np.uint32)
    bins = po.histo3d_bins(osc, d1, d2)
    ok = (bins != np.iinfo(np.uint64).max) & (d1 != d2)
    return d1[ok][:n], d2[ok][:n]


def gaussian_psf(fwhm=4.0, ks=0.5):
    sig = fwhm / 2.3548
    half = int(np.ceil(3 * sig / ks))
    x = (np.arange(2 * half + 1) - half) * ks
    k = np.exp(-0.5 * (x / sig) ** 2)
    k /= k.sum() * ks
    return 1e9, ks, k[None].astype(np.float32)


# ------------------------------------------------------------ integer work --
def test_histogram_maps_bitexact():
    sc, ip, p = make()
    d1, d2 = GOLD["d1"], GOLD["d2"]
    assert np.array_equal(yrt.histo3d_bins(sc, d1, d2), GOLD["bins"])
    a, b = yrt.histo3d_detpairs(sc, GOLD["query_bins"])
    assert np.array_equal(a, GOLD["query_d1"]) and np.array_equal(b, GOLD["query_d2"])
    rng = np.random.default_rng(2)
    x1 = rng.integers(0, sc.getNumDets(), 100000).astype(np.uint32)
    x2 = rng.integers(0, sc.getNumDets(), 100000).astype(np.uint32)
    osc = po.Scanner(*SC_ARGS)
    assert np.array_equal(yrt.histo3d_bins(sc, x1, x2), po.histo3d_bins(osc, x1, x2))
    allbins = np.arange(0, yrt.Histogram3D(sc).count(), 97, dtype=np.uint64)
    g1, g2 = yrt.histo3d_detpairs(sc, allbins)
    o1, o2 = po.histo3d_detpairs(osc, allbins)
    assert np.array_equal(g1, o1) and np.array_equal(g2, o2)


def test_histogram_maps_random_scanners_bitexact():
    # The device maps equal the oracle's on every bin and on random detector
    # pairs of the 25 random scanners whose properties (and agreement with the
    # reference library) tests/test_histo3d_props.py checks.
    from test_histo3d_props import SCANNERS, all_bins
    for i, o in enumerate(SCANNERS):
        sc = yrt.Scanner("r", o.axialFOV, o.crystalSize_z, o.crystalSize_trans,
                         o.crystalDepth, o.scannerRadius, o.detsPerRing, o.numRings,
                         o.numDOI, o.maxRingDiff, o.minAngDiff, o.detsPerBlock)
        bins = all_bins(o)
        g1, g2 = yrt.histo3d_detpairs(sc, bins)
        o1, o2 = po.histo3d_detpairs(o, bins)
        assert np.array_equal(g1, o1) and np.array_equal(g2, o2)
        rng = np.random.default_rng(100 + i)
        q1 = rng.integers(0, o.num_dets, 20000).astype(np.uint32)
        q2 = rng.integers(0, o.num_dets, 20000).astype(np.uint32)
        assert np.array_equal(yrt.histo3d_bins(sc, q1, q2), po.histo3d_bins(o, q1, q2))


def test_listmode_to_histogram_bitexact():
    sc, ip, p = make()
    d1, d2 = random_events(SC_ARGS, 300000, 3)
    lm = yrt.ListModeLUT(sc)
    lm.bind(d1, d2)
    h = yrt.convertToHistogram3D(lm)
    ref, bad = po.lm_to_histo3d(po.Scanner(*SC_ARGS), d1, d2)
    assert bad == 0
    assert np.array_equal(bits(h.data), bits(ref))


def test_listmode_to_histogram_rejects_invalid_pairs():
    sc, ip, p = make()
    # ring difference 15 is allowed, 16 rings: make a pair beyond mrd with a
    # smaller-mrd scanner.
    sc2 = yrt.Scanner("t", 64, 4, 4, 10, 300, 256, 16, 1, 3, 2, 1)
    lm = yrt.ListModeLUT(sc2)
    lm.bind(np.array([0, 5], np.uint32), np.array([128 + 256 * 10, 133], np.uint32))
    with pytest.raises(yrt.YrtbError, match="maximum ring difference"):
        yrt.convertToHistogram3D(lm)


# -------------------------------------------------------------- Siddon ----
def test_siddon_forward_golden():
    sc, ip, p = make()
    ev = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"])
    img = torch.from_numpy(GOLD["image"]).cuda()
    v = p.forward(img, ev).cpu().numpy()
    # Non-TOF mirror mode: every projection bit-identical to the reference.
    assert np.array_equal(bits(v), bits(GOLD["siddon_fwd"]))
    sc, ip, pt = make(tof=(214.0, 5))
    evt = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"], tof=GOLD["tof"])
    vt = pt.forward(img, evt).cpu().numpy()
    # TOF: same voxel sequence; the Gaussian uses the device expf (<= 2 ulp).
    assert rel_l2(vt, GOLD["siddon_tof_fwd"]) < 1e-6
    assert np.max(np.abs(vt - GOLD["siddon_tof_fwd"]) /
                  np.maximum(np.abs(GOLD["siddon_tof_fwd"]), 1e-30)) < 1e-5


def test_siddon_forward_lor_input_matches_detector_input():
    sc, ip, p = make()
    ev = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"])
    evl = yrt.DeviceEvents.from_arrays(lor=GOLD["lors"])
    img = torch.from_numpy(GOLD["image"]).cuda()
    assert torch.equal(p.forward(img, ev), p.forward(img, evl))


def test_siddon_backward_golden():
    sc, ip, p = make()
    ev = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"])
    vals = torch.from_numpy(GOLD["values"]).cuda()
    b = p.backward(vals, ev).cpu().numpy()
    assert rel_l2(b, GOLD["siddon_bwd"]) < 1e-6
    sc, ip, pt = make(tof=(214.0, 5))
    evt = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"], tof=GOLD["tof"])
    bt = pt.backward(vals, evt).cpu().numpy()
    assert rel_l2(bt, GOLD["siddon_tof_bwd"]) < 1e-5


@pytest.mark.parametrize("tof", [None, (214.0, 5), (95.0, 3), (214.0, 0)])
def test_siddon_random_vs_oracle(tof):
    sc_args = SC_ARGS
    ip_args = (64, 64, 32, 128, 128, 64)
    sc, ip, p = make(sc_args, ip_args, tof=tof)
    d1, d2 = random_events(sc_args, 40000, 7)
    rng = np.random.default_rng(8)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32) if tof else None
    img = rng.random(ip.shape, dtype=np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    lors, _ = po.lors_from_detpairs(po.scanner_lut(po.Scanner(*sc_args)), d1, d2)
    oip = po.ImageParams(*ip_args)
    pr = po.Proj(tof_fwhm_ps=tof[0] if tof else 0.0, tof_n_std=tof[1] if tof else 0)
    f32 = po.project(oip, pr, lors, image=img, tof=tv)
    f64 = po.project(oip, pr, lors, image=img, tof=tv, precision="f64")
    if tof is None:
        assert np.array_equal(bits(v), bits(f32))
    assert rel_l2(v, f32) < 1e-6
    assert rel_l2(v, f64) < 1e-5
    y = rng.random(len(d1)).astype(np.float32)
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    b64 = po.project(oip, pr, lors, values=y.astype(np.float64), tof=tv,
                     forward=False, precision="f64")
    # Image budget (1e-4); FP32 scatter of many small TOF-weighted terms.
    assert rel_l2(b, b64) < 1e-4
    b32 = po.project(oip, pr, lors, values=y, tof=tv, forward=False)
    assert rel_l2(b, b64) < 2 * rel_l2(b32, b64) + 1e-6
    # Adjoint identity of the device operator pair.
    lhs = float(np.dot(v.astype(np.float64), y))
    rhs = float(np.sum(b.astype(np.float64) * img))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def _walk_sequences(p, ev, n, cap=512):
    offs, wts, cnt = p.trace_walks(ev, cap)
    offs, wts, cnt = offs.cpu().numpy(), wts.cpu().numpy(), cnt.cpu().numpy()
    assert cnt.max() <= cap
    return [(offs[k, :cnt[k]], wts[k, :cnt[k]]) for k in range(n)]


@pytest.mark.parametrize("tof", [None, (214.0, 5)])
def test_walk_voxel_sequences_vs_oracle(tof):
    # The voxel index sequence of every walk, compared directly
    # (yrtb_trace_walks) with the CPU restatement's (orc_siddon_trace_f32 /
    # _f64).  Mirror arithmetic: the same sequence as the FP32 walk on every
    # ray, the non-TOF weights bit-identical, the TOF weights within 2e-6
    # (device expf).  Compensated arithmetic aims at the FP64 walk: it may
    # differ from it on no more rays than the mirror walk does, and on the
    # rays whose sequence matches, each interior weight (a difference of two
    # FP32 plane-crossing alphas times the LOR length L) is within 8 FP32
    # ulps of alpha times L (times the TOF kernel's peak with TOF) of FP64,
    # plus 1e-5 relative.  The first and last segments start or end where
    # the ray meets the FOV cylinder, a root of a quadratic that the FP32
    # set-up (the reference's) computes with cancellation near tangency:
    # they are held to 1e-4 L.  Random LORs plus LORs between opposite
    # crystals, which run on or near voxel planes.
    sc_args = SC_ARGS
    ip_args = (64, 64, 32, 128, 128, 64)
    osc = po.Scanner(*sc_args)
    d1, d2 = random_events(sc_args, 3000, 51)
    opp = np.arange(0, osc.num_dets, 7, dtype=np.uint32)
    d1 = np.concatenate([d1, opp])
    d2 = np.concatenate([d2, ((opp // 256) * 256 + (opp % 256 + 128) % 256).astype(np.uint32)])
    lors, _ = po.lors_from_detpairs(po.scanner_lut(osc), d1, d2)
    rng = np.random.default_rng(52)
    tv = rng.normal(0, 300, len(lors)).astype(np.float32) if tof else None
    oip = po.ImageParams(*ip_args)
    pr = po.Proj(tof_fwhm_ps=tof[0] if tof else 0.0, tof_n_std=tof[1] if tof else 0)
    n = len(lors)
    ev = yrt.DeviceEvents.from_arrays(lor=lors, tof=tv)
    seqs = {}
    for prec in (L.YRTB_MIRROR, L.YRTB_COMPENSATED):
        _, _, p = make(sc_args, ip_args, tof=tof, precision=prec)
        seqs[prec] = _walk_sequences(p, ev, n)
    f32 = [po.siddon_trace(oip, pr, lors[k], 0.0 if tv is None else float(tv[k]))
           for k in range(n)]
    f64 = [po.siddon_trace_f64(oip, pr, lors[k], 0.0 if tv is None else float(tv[k]))
           for k in range(n)]
    for k in range(n):
        o, w = seqs[L.YRTB_MIRROR][k]
        assert np.array_equal(o, f32[k][0]), k
        if tof:
            np.testing.assert_allclose(w, f32[k][1], rtol=2e-6, atol=0)
        else:
            assert np.array_equal(bits(w), bits(f32[k][1])), k
    differ = {prec: sum(1 for k in range(n) if not np.array_equal(seqs[prec][k][0], f64[k][0]))
              for prec in seqs}
    print(f"walks differing from the FP64 walk's sequence ({n} rays, tof={tof}): "
          f"mirror {differ[L.YRTB_MIRROR]}, compensated {differ[L.YRTB_COMPENSATED]}")
    assert differ[L.YRTB_COMPENSATED] <= differ[L.YRTB_MIRROR]
    peak = 1.0
    if tof:
        sigma = tof[0] * 0.299792458 / 2 / (2 * np.sqrt(2 * np.log(2)))
        peak = 1.0 / (np.sqrt(2 * np.pi) * sigma)
    for k in range(n):
        o, w = seqs[L.YRTB_COMPENSATED][k]
        if np.array_equal(o, f64[k][0]) and len(o):
            length = float(np.linalg.norm(lors[k, 3:].astype(np.float64) -
                                          lors[k, :3].astype(np.float64)))
            err = np.abs(w.astype(np.float64) - f64[k][1])
            bound = 8 * 2.0 ** -24 * length * peak + 1e-5 * np.abs(f64[k][1])
            bound[[0, -1]] = 1e-4 * length * peak
            j = int(np.argmax(err - bound))
            assert err[j] <= bound[j], (k, j, len(o), float(err[j]), float(bound[j]))


def test_siddon_image_offset_and_motion_and_frames():
    ip_args = (48, 40, 20, 120, 100, 80)
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*ip_args, 3.0, -2.0, 1.5, nt=3)
    pp = yrt.ProjectorParams(sc)
    p = yrt.DeviceProjector(sc, ip, pp)
    d1, d2 = random_events(SC_ARGS, 20000, 9)
    rng = np.random.default_rng(10)
    frames = rng.integers(-1, 3, len(d1)).astype(np.int32)
    from pyyrtpet_b200.synthetic import rigid_transforms
    xf = rigid_transforms(4, 11)
    mframe = rng.integers(-1, 4, len(d1)).astype(np.int32)
    img = rng.random(ip.shape, dtype=np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, frame=frames, motion_frame=mframe,
                                      motion=xf)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    # Oracle: apply the same rigid transform in float32 (Matrix * Vector3D
    # then + t, Matrix.cpp:177-186) and project into each event's frame.
    lut = po.scanner_lut(po.Scanner(*SC_ARGS))
    lors, _ = po.lors_from_detpairs(lut, d1, d2)
    f32 = np.float32
    moved = lors.copy()
    for i in np.nonzero(mframe >= 0)[0]:
        M = xf[mframe[i]].reshape(3, 4)
        R, t = M[:, :3], M[:, 3]
        for e in (0, 3):
            p_ = lors[i, e:e + 3]
            q = [f32(f32(f32(R[r, 0] * p_[0]) + f32(R[r, 1] * p_[1])) + f32(R[r, 2] * p_[2]))
                 for r in range(3)]
            moved[i, e:e + 3] = [f32(q[k] + t[k]) for k in range(3)]
    oip = po.ImageParams(*ip_args, 3.0, -2.0, 1.5, nt=3)
    ref = po.project(oip, po.Proj(), moved, image=img, frames=frames)
    assert np.array_equal(bits(v), bits(ref))
    assert np.all(v[frames < 0] == 0)


def test_multiray_vs_oracle_with_device_offsets():
    sc, ip, p = make(num_rays=4)
    d1, d2 = random_events(SC_ARGS, 5000, 12)
    rng = np.random.default_rng(13)
    img = rng.random(ip.shape, dtype=np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    offs = p.multiray_offsets(len(d1)).cpu().numpy()
    assert offs.shape == (len(d1), 12)
    assert np.all(np.abs(offs) <= 0.5)
    lut = po.scanner_lut(po.Scanner(*SC_ARGS))
    lors, ori = po.lors_from_detpairs(lut, d1, d2)
    pr = po.Proj(num_rays=4, crystal_z=4, crystal_trans=4)
    ref = po.project(po.ImageParams(*IP_ARGS), pr, lors, image=img,
                     orients=ori, ray_offsets=offs, precision="f64")
    assert rel_l2(v, ref) < 1e-5
    y = rng.random(len(d1)).astype(np.float32)
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    bref = po.project(po.ImageParams(*IP_ARGS), pr, lors, values=y.astype(np.float64),
                      orients=ori, ray_offsets=offs, forward=False,
                      precision="f64")
    assert rel_l2(b, bref) < 1e-5


def test_multiray_table_gives_the_same_projections():
    # yrtb_multiray_table: item indices below the table's size read their
    # offsets from it, the others still derive them from the generator; the
    # uniforms are the same, so the forward projections are bit-identical and
    # the EM image equal up to the order of the FP32 atomics.
    sc, ip, p = make(num_rays=4, tof=(214.0, 5))
    _, _, q = make(num_rays=4, tof=(214.0, 5))
    d1, d2 = random_events(SC_ARGS, 5000, 31)
    rng = np.random.default_rng(32)
    tof = rng.normal(0, 200, len(d1)).astype(np.float32)
    img = torch.from_numpy(rng.random(ip.shape, dtype=np.float32)).cuda()
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tof)
    v0 = p.forward(img, ev)
    e0 = p.em_step(img, torch.zeros(ip.shape, device="cuda"), ev)
    q.multiray_table(3000)
    assert torch.equal(q.forward(img, ev), v0)
    e1 = q.em_step(img, torch.zeros(ip.shape, device="cuda"), ev)
    assert rel_l2(e1.cpu().numpy(), e0.cpu().numpy()) < 1e-6
    q.multiray_table(len(d1))
    assert torch.equal(q.forward(img, ev), v0)


@pytest.mark.parametrize("tof,prec,rays", [(None, L.YRTB_MIRROR, 4),
                                           ((214.0, 5), L.YRTB_MIRROR, 4),
                                           ((214.0, 5), L.YRTB_COMPENSATED, 4),
                                           ((214.0, 5), L.YRTB_COMPENSATED, 3),
                                           (None, L.YRTB_COMPENSATED, 8)])
def test_multiray_one_lane_per_ray_matches_one_thread(tof, prec, rays):
    # One lane per ray (threads_per_lor = rays rounded up to a power of two,
    # the default with a table of offsets) adds the rays' forward sums in ray
    # order, as one thread walking the rays in turn does: the forward
    # projections are bit-identical; back projection and EM image equal up
    # to the order of the FP32 atomics, in each reduction mode the lanes use
    # (scalar, float4 groups, pairs).  Without a table covering the call,
    # the projector falls back to one thread per event.
    sc, ip, p = make(num_rays=rays, tof=tof, precision=prec)
    d1, d2 = random_events(SC_ARGS, 6000, 33)
    rng = np.random.default_rng(34)
    tv = rng.normal(0, 200, len(d1)).astype(np.float32) if tof else None
    img = torch.from_numpy(rng.random(ip.shape, dtype=np.float32)).cuda()
    y = torch.from_numpy(rng.uniform(0.1, 1.0, len(d1)).astype(np.float32)).cuda()
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    lanes = 1 << (rays - 1).bit_length()
    assert p.get_launch()["threads_per_lor"] == lanes
    v_gen = p.forward(img, ev)                 # no table yet: one thread per event
    p.multiray_table(len(d1))
    cfg = p.get_launch()
    out = {}
    for tpl, vg in ((1, 0), (lanes, 0), (lanes, 2), (lanes, 8)):
        cfg["threads_per_lor"] = tpl
        cfg["vector_groups"] = vg
        p.set_launch(**cfg)
        out[tpl, vg] = (p.forward(img, ev), p.backward(y, ev),
                        p.em_step(img, torch.zeros(ip.shape, device="cuda"), ev))
    base = out[1, 0]
    assert torch.equal(base[0], v_gen)
    for key, o in out.items():
        assert torch.equal(o[0], base[0]), key
        assert rel_l2(o[1].cpu().numpy(), base[1].cpu().numpy()) < 1e-6, key
        assert rel_l2(o[2].cpu().numpy(), base[2].cpu().numpy()) < 1e-6, key
    with pytest.raises(RuntimeError):
        cfg["threads_per_lor"] = 2 * lanes
        p.set_launch(**cfg)


# ------------------------------------------------------- tiled images ------
@pytest.mark.parametrize("tof,prec", [(None, L.YRTB_MIRROR), ((214.0, 5), L.YRTB_MIRROR),
                                      (None, L.YRTB_COMPENSATED),
                                      ((214.0, 5), L.YRTB_COMPENSATED)])
def test_tiled_image_layout_gives_the_same_projections(tof, prec):
    # YRTB_LAYOUT_TILE_4X2 changes only where each voxel is stored: the walks
    # visit the same voxels with the same weights in the same order, so the
    # forward projections are bit-identical to the row-major ones in every
    # vector mode; back projections and EM images agree up to the order of
    # the FP32 atomics.  Images with an offset and nt = 2 frames.
    ip_args = (32, 24, 16, 128, 96, 64, 1.5, -2.0, 3.0)
    sc, ip, p = make(ip_args=ip_args, tof=tof, precision=prec, nt=2)
    _, _, q = make(ip_args=ip_args, tof=tof, precision=prec, nt=2)
    d1, d2 = random_events(SC_ARGS, 8000, 41)
    rng = np.random.default_rng(42)
    tv = rng.normal(0, 200, len(d1)).astype(np.float32) if tof else None
    fr = rng.integers(0, 2, len(d1)).astype(np.int32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv, frame=torch.from_numpy(fr).cuda())
    img = torch.from_numpy(rng.random(ip.shape, dtype=np.float32)).cuda()
    y = torch.from_numpy(rng.uniform(0.1, 1.0, len(d1)).astype(np.float32)).cuda()
    T, R = L.YRTB_LAYOUT_TILE_4X2, L.YRTB_LAYOUT_ROW_MAJOR
    timg = q.to_layout(img, ip, T)
    assert torch.equal(q.to_layout(timg, ip, R), img.reshape(-1))
    assert not torch.equal(timg, img.reshape(-1))
    q.set_image_layout(T)
    assert q.get_image_layout() == T
    for vg in (0, 1, 2, 4):
        for h in (p, q):
            cfg = h.get_launch()
            cfg["vector_groups"] = vg
            h.set_launch(**cfg)
        f_row = p.forward(img, ev)
        f_tile = q.forward(timg.reshape(ip.shape), ev)
        assert torch.equal(f_row, f_tile), vg
        b_row = p.backward(y, ev)
        b_tile = q.to_layout(q.backward(y, ev), ip, R)
        assert rel_l2(b_tile.cpu().numpy(), b_row.cpu().numpy()) < 1e-6
        e_row = p.em_step(img, torch.zeros(ip.shape, device="cuda"), ev)
        e_tile = q.to_layout(q.em_step(timg.reshape(ip.shape),
                                       torch.zeros(ip.shape, device="cuda"), ev), ip, R)
        assert rel_l2(e_tile.cpu().numpy(), e_row.cpu().numpy()) < 1e-6


def test_tiled_image_layout_rejections():
    T = L.YRTB_LAYOUT_TILE_4X2
    for kw in (dict(projector="DD"), dict(num_rays=4),
               dict(ip_args=(30, 32, 16, 120, 128, 64)),
               dict(ip_args=(32, 31, 16, 128, 124, 64))):
        _, _, p = make(**kw)
        with pytest.raises(RuntimeError):
            p.set_image_layout(T)
    sc = yrt.Scanner("t", *SC_ARGS)
    pp = yrt.ProjectorParams(sc)
    pp.deterministic = True
    p = yrt.DeviceProjector(sc, yrt.ImageParams(*IP_ARGS), pp)
    with pytest.raises(RuntimeError):
        p.set_image_layout(T)
    with pytest.raises(RuntimeError):
        p.set_image_layout(7)


def test_osem_driver_tiles_internally_same_image():
    # yrtb_osem_listmode walks 4 x 2 tiles internally for a single-ray
    # Siddon projector set to that layout; its arguments and result stay
    # row-major.  The same OSEM driven subset by subset in row-major from
    # Python must agree (rel-L2 <= 1e-5: FP32 atomics order over 2 x 3
    # subset updates).
    import ctypes
    from pyyrtpet_b200.core import _stream
    sc, ip, q = make(tof=(214.0, 5), precision=L.YRTB_COMPENSATED)
    _, _, p = make(tof=(214.0, 5), precision=L.YRTB_COMPENSATED)
    q.set_image_layout(L.YRTB_LAYOUT_TILE_4X2)
    d1, d2 = random_events(SC_ARGS, 30000, 43)
    rng = np.random.default_rng(44)
    tv = rng.normal(0, 200, len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    sens = torch.from_numpy(rng.uniform(0.5, 2.0, ip.numVoxels).astype(np.float32)).cuda()
    sens[:100] = 0.0
    J, S = ip.numVoxels, 3
    x = torch.empty(J, device="cuda")
    work = torch.empty(2 * J, device="cuda")
    prm = L.yrtb_osem_params(2, S, 1.0, 1e-35, 1.19209e-07, 0, 0, None, None)
    L.check(L.lib().yrtb_osem_listmode(q.h, ctypes.byref(ev.c()), sens.data_ptr(),
                                       x.data_ptr(), work.data_ptr(), ctypes.byref(prm),
                                       _stream()))
    ref = torch.where(sens > 0, torch.full_like(sens, 0.125), torch.zeros_like(sens))
    sens_sub = (sens / S).contiguous()
    em = torch.empty(J, device="cuda")
    for _ in range(2):
        for s in range(S):
            em.zero_()
            p.em_step(ref, em, ev, rng=L.yrtb_range(s, S, 0))
            L.check(L.lib().yrtb_em_update(ref.data_ptr(), em.data_ptr(), sens_sub.data_ptr(),
                                           J, 1, 1, 1.19209e-07, None, _stream()))
    assert float(x.abs().sum()) > 0
    assert rel_l2(x.cpu().numpy(), ref.cpu().numpy()) < 1e-5


# ---------------------------------------------------------------- DD ------
@pytest.mark.parametrize("tof,psf,prec", [(None, False, L.YRTB_MIRROR),
                                          ((214.0, 5), False, L.YRTB_MIRROR),
                                          (None, True, L.YRTB_MIRROR),
                                          ((214.0, 5), True, L.YRTB_MIRROR),
                                          (None, True, L.YRTB_COMPENSATED),
                                          ((214.0, 5), True, L.YRTB_COMPENSATED)])
def test_dd_vs_oracle(tof, psf, prec):
    # Compensated DD + PSF takes the PSF integrals from prefix sums of the
    # kernel's trapezoid bins instead of the bin-by-bin loop.
    table = gaussian_psf() if psf else None
    sc, ip, p = make(projector="DD", tof=tof, psf=table, precision=prec)
    d1, d2 = random_events(SC_ARGS, 6000, 14)
    rng = np.random.default_rng(15)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32) if tof else None
    img = rng.random(ip.shape, dtype=np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    lut = po.scanner_lut(po.Scanner(*SC_ARGS))
    lors, ori = po.lors_from_detpairs(lut, d1, d2)
    pr = po.Proj(projector="DD", crystal_z=4, crystal_trans=4,
                 tof_fwhm_ps=tof[0] if tof else 0.0, tof_n_std=tof[1] if tof else 0,
                 psf_taps=table[2] if psf else None,
                 psf_s_step=table[0] if psf else 0, psf_k_spacing=table[1] if psf else 0)
    oip = po.ImageParams(*IP_ARGS)
    f32 = po.project(oip, pr, lors, image=img, orients=ori, tof=tv)
    f64 = po.project(oip, pr, lors, image=img, orients=ori, tof=tv, precision="f64")
    assert rel_l2(v, f32) < 1e-6
    assert rel_l2(v, f64) < 1e-5
    if tof is None and not psf:
        assert np.array_equal(bits(v), bits(f32))
    # Adjoint identity of the device operator pair.
    yv = rng.random(len(d1)).astype(np.float32)
    bv = p.backward(torch.from_numpy(yv).cuda(), ev).cpu().numpy()
    lhs = float(np.dot(v.astype(np.float64), yv))
    rhs = float(np.sum(bv.astype(np.float64) * img))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    y = rng.random(len(d1)).astype(np.float32)
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    b64 = po.project(oip, pr, lors, values=y.astype(np.float64), orients=ori,
                     tof=tv, forward=False, precision="f64")
    assert rel_l2(b, b64) < 1e-5


def test_dd_golden_bitexact():
    sc, ip, p = make(projector="DD")
    ev = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"])
    v = p.forward(torch.from_numpy(GOLD["image"]).cuda(), ev).cpu().numpy()
    assert np.array_equal(bits(v), bits(GOLD["dd_fwd"]))


# ------------------------------------------------------------ EM / OSEM ---
def test_em_step_vs_oracle_f64():
    sc, ip, p = make(tof=(214.0, 5))
    d1, d2 = random_events(SC_ARGS, 30000, 16)
    rng = np.random.default_rng(17)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32)
    sens = rng.uniform(0.5, 1.5, len(d1)).astype(np.float32)
    att = rng.uniform(0.2, 1.0, len(d1)).astype(np.float32)
    add = rng.uniform(0.0, 0.05, len(d1)).astype(np.float32)
    img = rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv, sens=sens, att=att,
                                      additive=add)
    em = torch.zeros(ip.shape, device="cuda")
    p.em_step(torch.from_numpy(img).cuda(), em, ev, global_scale=1.3)
    lors, _ = po.lors_from_detpairs(po.scanner_lut(po.Scanner(*SC_ARGS)), d1, d2)
    ref = po.em_step_f64(po.ImageParams(*IP_ARGS), po.Proj(tof_fwhm_ps=214.0, tof_n_std=5),
                         lors, img, tof=tv, sens=sens, att=att, additive=add,
                         global_scale=1.3)
    assert rel_l2(em.cpu().numpy(), ref) < 1e-4


def _small_c1_problem(n=60000, seed=18, tof=False):
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    ev = S.generate_events(sc, n, seed, tof_fwhm_ps=214.0 if tof else None)
    return sc, ip, ev


@needs_ref
@pytest.mark.parametrize("tof", [False, True])
def test_sensitivity_and_listmode_osem_vs_reference(tof):
    sc, ip, evs = _small_c1_problem(tof=tof)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 3
    osem.setListModeEnabled(True)
    if tof:
        osem.addTOF(214.0, 5)
    sens = osem.generateSensitivityImages()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    rs, _ = po.ref_sensitivity(osc, oip, listmode=True)
    assert rel_l2(sens[0].cpu().numpy(), rs[0]) < 1e-5
    e = evs.numpy()
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e.get("tof"))
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"],
                                  tof=e.get("tof"), iterations=2, subsets=3,
                                  tof_fwhm_ps=214.0 if tof else 0.0,
                                  tof_n_std=5 if tof else 0)
    assert rel_l2(img, ref) < 1e-4


@needs_ref
def test_listmode_osem_with_corrections_vs_reference():
    from pyyrtpet_b200 import synthetic as S
    sc, ip, evs = _small_c1_problem(n=40000, seed=19, tof=True)
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    h = yrt.Histogram3D(sc)
    eff = S.crystal_efficiencies(sc, 20).numpy()
    allb = np.arange(h.count(), dtype=np.uint64)
    a, b = yrt.histo3d_detpairs(sc, allb)
    h.data = (eff[a] * eff[b]).astype(np.float32)
    mu_ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    mu = S.Phantom(cyl_half_length=32).mu_image(mu_ip).numpy()
    e = evs.numpy()
    rng = np.random.default_rng(21)
    randoms = rng.uniform(0.0, 0.01, len(e["d1"])).astype(np.float32)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 2
    osem.setListModeEnabled(True)
    osem.addTOF(214.0, 5)
    osem.setSensitivityHistogram(h)
    osem.setAttenuationImage(mu, mu_ip)
    sens = osem.generateSensitivityImages()
    rs, _ = po.ref_sensitivity(osc, oip, listmode=True, sens_histo=h.data,
                               att_params=oip, att_image=mu)
    assert rel_l2(sens[0].cpu().numpy(), rs[0]) < 1e-5
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e["tof"], randoms=randoms)
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"],
                                  tof=e["tof"], randoms=randoms,
                                  sens_histo=h.data, att_params=oip,
                                  att_image=mu, iterations=2, subsets=2,
                                  tof_fwhm_ps=214.0, tof_n_std=5)
    assert rel_l2(img, ref) < 1e-4


@needs_ref
def test_histogram_osem_dd_psf_vs_reference(tmp_path):
    from pyyrtpet_b200 import synthetic as S
    sc, ip, evs = _small_c1_problem(n=200000, seed=22)
    lm = yrt.ListModeLUT(sc)
    e = evs.numpy()
    lm.bind(e["d1"], e["d2"])
    hist = yrt.convertToHistogram3D(lm)
    s_step, ks, taps = gaussian_psf()
    csv = str(tmp_path / "psf.csv")
    yrt.write_psf_csv(csv, s_step, ks, taps)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 1
    osem.num_OSEM_subsets = 4
    osem.setProjector("DD")
    osem.addProjPSF(csv)
    osem.setDataInput(hist)
    sens = osem.generateSensitivityImages()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    rs, _ = po.ref_sensitivity(osc, oip, projector="DD", subsets=4,
                               listmode=False, psf_csv=csv)
    for s in range(4):
        assert rel_l2(sens[s].cpu().numpy(), rs[s]) < 1e-5
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_histo3d(osc, oip, rs, hist.data, psf_csv=csv,
                                 projector="DD", iterations=1, subsets=4)
    # The reference CPU back projector uses flipped PSF taps for A^T
    # (ProjectorDD.cpp:278-283); so does this path.
    assert rel_l2(img, ref) < 1e-4


@pytest.mark.parametrize("projector,rays,det", [("S", 1, False), ("S", 4, False),
                                                ("DD", 1, False), ("DDPSF", 1, False),
                                                ("DDPSF", 1, True)])
def test_histogram_em_over_nonzero_bin_list(projector, rays, det):
    # yrtb_histo3d_subset_nonzero selects exactly the bins the full-subset
    # pass does work for (BinIteratorRangeHistogram3D order, valid pair,
    # m != 0), and the pass over that list gives the full pass's image
    # (bit-identical in deterministic mode, 1e-6 rel-L2 otherwise: the same
    # FP32 terms reduced in another order).
    psf = gaussian_psf() if projector == "DDPSF" else None
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*IP_ARGS)
    pp = yrt.ProjectorParams(sc)
    pp.setProjector("S" if projector == "S" else "DD")
    pp.numRays = rays
    if psf is not None:
        pp.setProjPsf(*psf)
    pp.deterministic = det
    p = yrt.DeviceProjector(sc, ip, pp)
    h = yrt.Histogram3D(sc)
    rng = np.random.default_rng(41)
    m = np.where(rng.random(h.histoSize) < 0.1,
                 rng.integers(1, 5, h.histoSize), 0).astype(np.float32)
    meas = torch.from_numpy(m).cuda()
    img = torch.from_numpy(rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)).cuda()
    S = 5
    for s in (0, 3):
        nps = h.numPhi // S + (1 if s + (h.numPhi // S) * S < h.numPhi else 0)
        count = h.numR * nps * h.numZBin
        k = np.arange(count, dtype=np.uint64)
        per = np.uint64(nps * h.numR)
        z, rem = k // per, k % per
        phi = (rem // np.uint64(h.numR)) * np.uint64(S) + np.uint64(s)
        b = z * np.uint64(h.numPhi * h.numR) + phi * np.uint64(h.numR) + rem % np.uint64(h.numR)
        a1, a2 = yrt.histo3d_detpairs(sc, b)
        want = k[(m[b] != 0) & ~((a1 == 0) & (a2 == 0))]
        got = p.histo3d_subset_nonzero(meas, S, s, count)
        assert np.array_equal(got.cpu().numpy().view(np.uint64), want)
        full = torch.zeros(ip.shape, device="cuda")
        p.em_step_histo3d(img, full, meas, S, s)
        lst = torch.zeros(ip.shape, device="cuda")
        p.em_step_histo3d(img, lst, meas, S, s, bins=got)
        if det:
            assert torch.equal(lst, full)
        else:
            assert rel_l2(lst.cpu().numpy(), full.cpu().numpy()) < 1e-6
    with pytest.raises(yrt.YrtbError, match="capacity"):
        p.histo3d_subset_nonzero(meas, S, 0, 10)


def test_histogram_dd_psf_compensated_rows_split_over_threads():
    # Compensated DD + PSF histogram EM runs 4 threads per bin, each on a share
    # of the bin's rows, the forward partial sums added over the group.  Its
    # image equals the single-thread compensated pass (deterministic mode,
    # fixed-point sums) to 1e-6 and the mirror pass to 1e-5.
    psf = gaussian_psf()
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*IP_ARGS)
    h = yrt.Histogram3D(sc)
    rng = np.random.default_rng(43)
    m = np.where(rng.random(h.histoSize) < 0.05,
                 rng.integers(1, 5, h.histoSize), 0).astype(np.float32)
    meas = torch.from_numpy(m).cuda()
    img = torch.from_numpy(rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)).cuda()
    out = {}
    for name, prec, det in (("split", L.YRTB_COMPENSATED, False),
                            ("single", L.YRTB_COMPENSATED, True),
                            ("mirror", L.YRTB_MIRROR, False)):
        pp = yrt.ProjectorParams(sc)
        pp.setProjector("DD")
        pp.setProjPsf(*psf)
        pp.precision = prec
        pp.deterministic = det
        p = yrt.DeviceProjector(sc, ip, pp)
        em = torch.zeros(ip.shape, device="cuda")
        for s in range(3):
            p.em_step_histo3d(img, em, meas, 3, s)
        out[name] = em.cpu().numpy()
    assert np.count_nonzero(out["split"]) > 0
    assert rel_l2(out["split"], out["single"]) < 1e-6
    assert rel_l2(out["split"], out["mirror"]) < 1e-5


def test_graph_and_plain_osem_agree():
    sc, ip, evs = _small_c1_problem(n=30000, seed=23, tof=True)
    e = evs.numpy()
    outs = []
    for graphs in (False, True):
        osem = yrt.createOSEM(sc)
        osem.setImageParams(ip)
        osem.num_MLEM_iterations = 2
        osem.num_OSEM_subsets = 3
        osem.setListModeEnabled(True)
        osem.addTOF(214.0, 5)
        osem.useGraphs = graphs
        osem.generateSensitivityImages()
        lm = yrt.ListModeLUT(sc)
        lm.bind(e["d1"], e["d2"], tof=e["tof"])
        osem.setDataInput(lm)
        outs.append(osem.reconstruct().cpu().numpy())
    assert rel_l2(outs[0], outs[1]) < 1e-5


@needs_ref
def test_crystal_factor_sensitivity_and_gather_equal_histogram_forms():
    # LOR sensitivity formed in the kernel as eff[d1] * eff[d2] against a
    # sensitivity histogram holding those products (filled through the
    # reference's own bin -> detector-pair map): the per-event gather is
    # bit-identical, and so is the sensitivity image in deterministic mode;
    # the image also matches the reference's sensitivity image (1e-5).
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    osc = po.Scanner(*SC_ARGS)
    eff = S.crystal_efficiencies(sc, 23)
    h = po.ref_histo3d_crystal_product(osc, eff.numpy())
    a, b = yrt.histo3d_detpairs(sc, np.arange(len(h), dtype=np.uint64))
    assert np.array_equal(bits(h), bits(eff.numpy()[a] * eff.numpy()[b]))
    pp = yrt.ProjectorParams(sc)
    pp.deterministic = True
    p = yrt.DeviceProjector(sc, ip, pp)
    eff_d, h_d = eff.cuda(), torch.from_numpy(h).cuda()
    s_eff = p.sensitivity_histo3d(torch.zeros(ip.shape, device="cuda"),
                                  crystal_eff=eff_d)
    s_hist = p.sensitivity_histo3d(torch.zeros(ip.shape, device="cuda"),
                                   sens_histo=h_d)
    assert torch.equal(s_eff, s_hist)
    rs, _ = po.ref_sensitivity(osc, po.ImageParams(32, 32, 16, 256, 256, 128),
                               listmode=True, sens_histo=h)
    got = s_eff.cpu().numpy()
    got[got <= 1.0] = 0.0  # the reference's hard threshold (1.0)
    assert rel_l2(got, rs[0]) < 1e-5
    d1, d2 = random_events(SC_ARGS, 20000, 24)
    ev = yrt.DeviceEvents.from_arrays(d1, d2)
    g_eff = p.gather_crystal_product(eff_d, ev)
    g_hist = p.gather_histo3d(h_d, ev)
    assert torch.equal(g_eff, g_hist)


def test_em_update_variants_vs_numpy():
    rng = np.random.default_rng(24)
    J, nt = 1000, 3
    x = rng.uniform(0.1, 2, (nt, J)).astype(np.float32)
    u = rng.uniform(0.1, 2, (nt, J)).astype(np.float32)
    s = rng.uniform(-0.1, 2, J).astype(np.float32)
    c = np.array([0.5, 1.0, 2.0], np.float32)
    xt = torch.from_numpy(x.copy()).cuda()
    ut, st, ct = (torch.from_numpy(a).cuda() for a in (u, s, c))
    L.check(L.lib().yrtb_em_update(xt.data_ptr(), ut.data_ptr(), st.data_ptr(),
                                   J, nt, 1, 1.19209e-07, ct.data_ptr(), None))
    torch.cuda.synchronize()
    ref = x.copy()
    for r in range(nt):
        inv_c = np.float32(1) / c[r]
        m = s > np.float32(1.19209e-07) * inv_c
        ref[r, m] *= (u[r, m] * inv_c) / s[m]
    np.testing.assert_allclose(xt.cpu().numpy(), ref, rtol=1e-6)


@pytest.mark.parametrize("J", [4096, 1001])  # float4 form, scalar form
@pytest.mark.parametrize("mode", ["broadcast", "per_frame", "scaled"])
def test_em_update_modes_bit_exact(J, mode):
    # Image::updateEMThreshold{Static,Dynamic,DynamicWithScaling,
    # DynamicWith4DSens} (Image.cpp:651-833): x *= u / s where s > thr, the
    # same FP32 operations as numpy's, so the results are bit-identical.
    rng = np.random.default_rng(31)
    nt = 5
    thr = np.float32(1.19209e-07)
    x = rng.uniform(0.1, 2, (nt, J)).astype(np.float32)
    u = rng.uniform(0.1, 2, (nt, J)).astype(np.float32)
    sens_nt = nt if mode == "per_frame" else 1
    s = rng.uniform(-0.1, 2, (sens_nt, J)).astype(np.float32)
    s[:, ::7] = 0.0
    c = rng.uniform(0.5, 2, nt).astype(np.float32)
    xt = torch.from_numpy(x.copy()).cuda()
    ut, st, ct = (torch.from_numpy(a).cuda() for a in (u, s, c))
    L.check(L.lib().yrtb_em_update(xt.data_ptr(), ut.data_ptr(), st.data_ptr(), J, nt,
                                   sens_nt, thr,
                                   ct.data_ptr() if mode == "scaled" else None, None))
    torch.cuda.synchronize()
    ref = x.copy()
    for r in range(nt):
        sr = s[r] if mode == "per_frame" else s[0]
        if mode == "scaled":
            inv_c = np.float32(1) / c[r]
            m = sr > thr * inv_c
            ref[r, m] *= (u[r, m] * inv_c) / sr[m]
        else:
            m = sr > thr
            ref[r, m] *= u[r, m] / sr[m]
    assert np.array_equal(xt.cpu().numpy(), ref)


@pytest.mark.parametrize("J", [4096, 1001])
@pytest.mark.parametrize("broadcast", [1, 0])
def test_apply_threshold_bit_exact(J, broadcast):
    # Image::applyThreshold[Broadcast] (Image.cpp:595-650): x = m <= thr ? x*les + leo
    # : x*gts + gto, FP32 products and sums without contraction.
    rng = np.random.default_rng(32)
    nt = 3
    x = rng.uniform(-1, 2, (nt, J)).astype(np.float32)
    m = rng.uniform(-0.5, 1, (1 if broadcast else nt, J)).astype(np.float32)
    a = [np.float32(v) for v in (0.25, 0.0, 1.5, -0.125, 0.5)]  # thr les leo gts gto
    xt = torch.from_numpy(x.copy()).cuda()
    mt = torch.from_numpy(m).cuda()
    L.check(L.lib().yrtb_apply_threshold(xt.data_ptr(), mt.data_ptr(), J, nt, broadcast,
                                         *a, None))
    torch.cuda.synchronize()
    mm = np.broadcast_to(m, x.shape)
    ref = np.where(mm <= a[0], x * a[1] + a[2], x * a[3] + a[4]).astype(np.float32)
    assert np.array_equal(xt.cpu().numpy(), ref)


# ------------------------------------------------------------- errors -----
def test_invalid_detector_ids_are_counted_not_read():
    sc, ip, p = make()
    ev = yrt.DeviceEvents.from_arrays(np.array([0, 10**6], np.uint32),
                                      np.array([128, 5], np.uint32))
    v = p.forward(torch.ones(ip.shape, device="cuda"), ev).cpu().numpy()
    assert v[1] == 0
    assert p.take_event_errors() == 1


def test_tof_projector_requires_tof_values():
    sc, ip, p = make(tof=(214.0, 5))
    ev = yrt.DeviceEvents.from_arrays(GOLD["d1"], GOLD["d2"])
    with pytest.raises(yrt.YrtbError, match="TOF"):
        p.forward(torch.ones(ip.shape, device="cuda"), ev)


def test_event_ordering_is_subset_major_permutation():
    sc, ip, p = make(tof=(214.0, 5))
    d1, d2 = random_events(SC_ARGS, 50001, 25)
    rng = np.random.default_rng(26)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    out, offs = p.order_events(ev, 7)
    perm = out.perm.cpu().numpy()
    n = len(d1)
    assert np.array_equal(np.sort(perm), np.arange(n))
    for s in range(7):
        src = perm[offs[s]:offs[s + 1]]
        assert np.all(src % 7 == s)
        assert len(src) == len(range(s, n, 7))
    assert np.array_equal(out.d1.cpu().numpy().view(np.uint32), d1[perm])
    assert np.array_equal(out.tof.cpu().numpy(), tv[perm])
    # Same EM image for the subset whatever the event order.
    img = torch.from_numpy(rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)).cuda()
    em_a = torch.zeros(ip.shape, device="cuda")
    em_b = torch.zeros(ip.shape, device="cuda")
    p.em_step(img, em_a, ev, rng=L.yrtb_range(3, 7, 0))
    p.em_step(img, em_b, out, rng=L.yrtb_range(int(offs[3]), 1, int(offs[4] - offs[3])))
    assert rel_l2(em_b.cpu().numpy(), em_a.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("first", [0, 3, 10**9 + 5])
def test_event_ordering_of_a_shard_keeps_global_subsets(first):
    # A shard whose first event has global index `first`: local event e is
    # in subset (first + e) mod S; the subset-major order and its offsets
    # follow that rule, and a shard's EM pass over a subset equals the pass
    # over the same events of the whole stream.
    from pyyrtpet_b200.distributed import local_subset_range
    sc, ip, p = make(tof=(214.0, 5))
    d1, d2 = random_events(SC_ARGS, 30003, 27)
    rng = np.random.default_rng(28)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    S = 7
    out, offs = p.order_events(ev, S, first_global_index=first)
    perm = out.perm.cpu().numpy()
    n = len(d1)
    assert np.array_equal(np.sort(perm), np.arange(n))
    img = torch.from_numpy(rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)).cuda()
    for s in range(S):
        src = perm[offs[s]:offs[s + 1]]
        assert np.all((first + src) % S == s)
        start, stride, count = local_subset_range(n, first, S, s)
        assert count == len(src)
        if s == 2:
            em_a = torch.zeros(ip.shape, device="cuda")
            em_b = torch.zeros(ip.shape, device="cuda")
            p.em_step(img, em_a, ev, rng=L.yrtb_range(start, stride, count))
            p.em_step(img, em_b, out, rng=L.yrtb_range(int(offs[s]), 1, count))
            assert rel_l2(em_b.cpu().numpy(), em_a.cpu().numpy()) < 1e-5


@needs_ref
@pytest.mark.parametrize("grid", [(32, 32, 16, 256, 256, 128), (64, 64, 32, 256, 256, 128)])
def test_attenuation_factors_mirror_equal_reference_fp32(grid):
    # Mirror arithmetic reproduces the reference's FP32 Siddon projection of
    # the mu-map (Corrector::getAttenuationFactorFromAttenuationImage) walk
    # for walk: the factors differ at most by the last bits of exp.  (A walk
    # limited to the mu-map's support box started on a different first
    # segment and put whole walks one voxel off: up to 19 % on a factor.)
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(*grid)
    pp = yrt.ProjectorParams(sc)
    pp.precision = L.YRTB_MIRROR
    p = yrt.DeviceProjector(sc, ip, pp)
    e = S.generate_events(sc, 50000, 62).numpy()
    mu = S.Phantom(cyl_half_length=32).mu_image(ip).numpy()
    ev = yrt.DeviceEvents.from_arrays(e["d1"], e["d2"])
    acf = p.attenuation_factors(torch.from_numpy(mu).cuda().reshape(-1), ip, ev).cpu().numpy()
    osc = po.Scanner(*SC_ARGS)
    lors, _ = po.lors_from_detpairs(po.scanner_lut(osc), e["d1"], e["d2"])
    line = po.ref_siddon(osc, po.ImageParams(*grid), lors, image=mu)
    line = line[0] if isinstance(line, tuple) else line
    ref = np.exp(np.float32(-0.1) * line.astype(np.float32)).astype(np.float32)
    assert np.max(np.abs(acf - ref) / ref) < 1e-6


@pytest.mark.parametrize("precision", [L.YRTB_MIRROR, L.YRTB_COMPENSATED])
@pytest.mark.parametrize("support", ["cylinder", "offcentre", "empty"])
def test_attenuation_factors_vs_oracle(support, precision):
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(64, 64, 32, 256, 256, 128)
    pp = yrt.ProjectorParams(sc)
    pp.precision = precision
    p = yrt.DeviceProjector(sc, ip, pp)
    evs = S.generate_events(sc, 30000, 91)
    e = evs.numpy()
    mu = S.Phantom(cyl_half_length=32).mu_image(ip).numpy()
    if support == "offcentre":
        mu = np.zeros_like(mu)
        mu[0, 3:9, 40:52, 10:20] = 0.15
    elif support == "empty":
        mu = np.zeros_like(mu)
    ev = yrt.DeviceEvents.from_arrays(e["d1"], e["d2"])
    acf = p.attenuation_factors(torch.from_numpy(mu).cuda().reshape(-1), ip, ev).cpu().numpy()
    lut = po.scanner_lut(po.Scanner(*SC_ARGS))
    lors, _ = po.lors_from_detpairs(lut, e["d1"], e["d2"])
    line = po.project(po.ImageParams(64, 64, 32, 256, 256, 128), po.Proj(), lors,
                      image=mu, precision="f64")
    ref = np.exp(-0.1 * line)
    if support == "empty":
        assert np.all(acf == 1.0)
    assert rel_l2(acf, ref) < 1e-6
    assert np.max(np.abs(acf - ref) / ref) < 1e-5
