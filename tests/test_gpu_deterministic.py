"""Deterministic two-pass back projection (64-bit fixed-point scatter).

Checks, through the C ABI: results bit-identical across repeated calls and
across permutations of the events (the float-atomic path is order
dependent); within 1e-5 relative L2 of the FP64 oracle and no worse than
the float-atomic path (the accumulation is exact to ~2^-40 of the largest
contribution; the FP32 weights remain); OSEM with graphs and without
bit-identical; a NaN value makes the whole image NaN instead of a silently
wrong sum.
"""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L

pytestmark = pytest.mark.gpu

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
IP_ARGS = (32, 32, 16, 128, 128, 64)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(projector="S", tof=None, num_rays=1, precision=L.YRTB_COMPENSATED,
         deterministic=True, ip_args=IP_ARGS, nt=1):
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*ip_args, nt=nt)
    pp = yrt.ProjectorParams(sc)
    pp.setProjector(projector)
    pp.numRays = num_rays
    pp.precision = precision
    pp.deterministic = deterministic
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


CASES = [("S", None, 1, L.YRTB_MIRROR), ("S", (214.0, 5), 1, L.YRTB_COMPENSATED),
         ("S", (214.0, 5), 1, L.YRTB_MIRROR), ("S", None, 4, L.YRTB_COMPENSATED),
         ("DD", None, 1, L.YRTB_MIRROR), ("DD", (214.0, 5), 1, L.YRTB_MIRROR)]


@pytest.mark.parametrize("projector,tof,rays,prec", CASES)
def test_backward_bit_identical_under_permutation(projector, tof, rays, prec):
    sc, ip, p = make(projector, tof, rays, prec)
    d1, d2 = random_events(40000, 31)
    rng = np.random.default_rng(32)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32) if tof else None
    y = rng.random(len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    a = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if rays == 1:
        # Multi-ray offsets follow the event's index in the batch, so only the
        # single-ray projectors are permutation invariant by definition.
        perm = rng.permutation(len(d1))
        evp = yrt.DeviceEvents.from_arrays(d1[perm], d2[perm],
                                           tof=None if tv is None else tv[perm])
        c = p.backward(torch.from_numpy(y[perm]).cuda(), evp).cpu().numpy()
        assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
    # Same operator as the float-atomic path (image budget 1e-4; the two
    # differ only by the float path's accumulation error).
    _, _, pf = make(projector, tof, rays, prec, deterministic=False)
    f = pf.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    assert rel_l2(a, f) < 1e-5


@pytest.mark.parametrize("tof", [None, (214.0, 5)])
def test_backward_vs_oracle_f64(tof):
    sc, ip, p = make("S", tof, 1, L.YRTB_COMPENSATED)
    d1, d2 = random_events(40000, 33)
    rng = np.random.default_rng(34)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32) if tof else None
    y = rng.random(len(d1)).astype(np.float32)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    lors, _ = po.lors_from_detpairs(po.scanner_lut(po.Scanner(*SC_ARGS)), d1, d2)
    pr = po.Proj(tof_fwhm_ps=tof[0] if tof else 0.0, tof_n_std=tof[1] if tof else 0)
    b64 = po.project(po.ImageParams(*IP_ARGS), pr, lors, values=y.astype(np.float64),
                     tof=tv, forward=False, precision="f64")
    # Fixed-point sums are exact to ~n * 2^-61 of the largest term; what is
    # left is the FP32 weights (FP32 alpha arithmetic of the walk) and the
    # final rounding to float: within the 1e-5 projection budget, and no
    # worse than the float-atomic path.
    err = rel_l2(b, b64)
    assert err < 1e-5
    _, _, pf = make("S", tof, 1, L.YRTB_COMPENSATED, deterministic=False)
    bf = pf.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    assert err <= rel_l2(bf, b64) * 1.001 + 1e-8


def test_em_step_deterministic_and_vs_oracle_f64():
    sc, ip, p = make("S", (214.0, 5), 1, L.YRTB_COMPENSATED)
    d1, d2 = random_events(30000, 35)
    rng = np.random.default_rng(36)
    tv = rng.normal(0, 300, len(d1)).astype(np.float32)
    sens = rng.uniform(0.5, 1.5, len(d1)).astype(np.float32)
    att = rng.uniform(0.2, 1.0, len(d1)).astype(np.float32)
    add = rng.uniform(0.0, 0.05, len(d1)).astype(np.float32)
    img = rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)
    gimg = torch.from_numpy(img).cuda()

    def run(proj, perm):
        ev = yrt.DeviceEvents.from_arrays(d1[perm], d2[perm], tof=tv[perm],
                                          sens=sens[perm], att=att[perm],
                                          additive=add[perm])
        em = torch.zeros(ip.shape, device="cuda")
        proj.em_step(gimg, em, ev, global_scale=1.3)
        return em.cpu().numpy()

    ident = np.arange(len(d1))
    a = run(p, ident)
    b = run(p, ident)
    c = run(p, rng.permutation(len(d1)))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
    lors, _ = po.lors_from_detpairs(po.scanner_lut(po.Scanner(*SC_ARGS)), d1, d2)
    ref = po.em_step_f64(po.ImageParams(*IP_ARGS), po.Proj(tof_fwhm_ps=214.0, tof_n_std=5),
                         lors, img, tof=tv, sens=sens, att=att, additive=add,
                         global_scale=1.3)
    # Image budget 1e-4 (the float-atomic path's own test uses the same).
    err = rel_l2(a, ref)
    assert err < 1e-4
    _, _, pf = make("S", (214.0, 5), 1, L.YRTB_COMPENSATED, deterministic=False)
    assert err <= rel_l2(run(pf, ident), ref) * 1.001 + 1e-8


def test_nan_value_poisons_the_image():
    sc, ip, p = make("S", None, 1, L.YRTB_MIRROR)
    d1, d2 = random_events(1000, 37)
    y = np.ones(len(d1), np.float32)
    y[10] = np.nan
    ev = yrt.DeviceEvents.from_arrays(d1, d2)
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    assert np.isnan(b).all()
    z = p.backward(torch.zeros(len(d1), device="cuda"), ev).cpu().numpy()
    assert not z.any()


def test_histogram_sensitivity_and_em_deterministic():
    sc, ip, p = make("DD", None, 1, L.YRTB_MIRROR)
    _, _, pf = make("DD", None, 1, L.YRTB_MIRROR, deterministic=False)
    h = yrt.Histogram3D(sc)
    rng = np.random.default_rng(38)
    meas = torch.from_numpy(rng.poisson(0.3, h.count()).astype(np.float32)).cuda()
    sh = torch.from_numpy(rng.uniform(0.5, 1.5, h.count()).astype(np.float32)).cuda()
    outs = []
    for proj in (p, p, pf):
        s = torch.zeros(ip.shape, device="cuda")
        proj.sensitivity_histo3d(s, num_subsets=8, subset=3, sens_histo=sh)
        em = torch.zeros(ip.shape, device="cuda")
        x = torch.full(ip.shape, 1.0, device="cuda")
        proj.em_step_histo3d(x, em, meas, 8, 3, sens_histo=sh)
        outs.append((s.cpu().numpy(), em.cpu().numpy()))
    for k in range(2):
        assert np.array_equal(outs[0][k].view(np.uint32), outs[1][k].view(np.uint32))
        assert rel_l2(outs[0][k], outs[2][k]) < 1e-5


def test_osem_deterministic_graph_and_plain_bit_identical():
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    e = S.generate_events(sc, 30000, 39, tof_fwhm_ps=214.0).numpy()
    outs = []
    for graphs in (False, True, True):
        osem = yrt.createOSEM(sc)
        osem.setImageParams(ip)
        osem.num_MLEM_iterations = 2
        osem.num_OSEM_subsets = 3
        osem.setListModeEnabled(True)
        osem.addTOF(214.0, 5)
        osem.projectorParams.precision = L.YRTB_COMPENSATED
        osem.projectorParams.deterministic = True
        osem.useGraphs = graphs
        osem.generateSensitivityImages()
        lm = yrt.ListModeLUT(sc)
        lm.bind(e["d1"], e["d2"], tof=e["tof"])
        osem.setDataInput(lm)
        outs.append(osem.reconstruct().cpu().numpy())
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    assert np.array_equal(outs[1].view(np.uint32), outs[2].view(np.uint32))
