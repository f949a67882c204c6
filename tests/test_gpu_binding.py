"""The reference's own drivers running on libyrtb through the binding classes.

yrt-pet_b200/binding/yrtb_yrtpet.cu subclasses YRT-PET's
OperatorProjectorDevice (OperatorProjectorB200) and OSEM_GPU (OSEM_GPU_B200)
so that the reference's C++ code calls libyrtb: its OperatorProjectorDevice::
applyA / applyAH staging and batching (src/operators/OperatorProjectorDevice.cu:
442-706), and its OSEM::reconstruct (src/recon/OSEM.cpp:315-365) with the
corrector, batch loading and sensitivity images of OSEM_GPU.  The test
harness (oracle/ref_harness.cpp built with REF_HARNESS_B200) runs them on
the same inputs as the reference's own GPU path (the REF_HARNESS_GPU build)
and as libyrtb's own drivers.

Tolerances: forward projections through the binding equal libyrtb's own
projections of the same detector pairs bit for bit (the rows carry the
reference's LOR endpoints, which equal libyrtb's LUT); against the reference
GPU projector 1e-5 rel-L2 per projection; images 1e-4 rel-L2 against the
reference's GPU reconstruction (mirror arithmetic).
"""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (po.ref_b200_available() and
                                      po.ref_gpu_available()),
                                 reason="binding harness not built")]

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
IP_ARGS = (48, 48, 24, 192, 192, 96, 3.0, 10.0, -15.0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def random_events(n, seed):
    rng = np.random.default_rng(seed)
    osc = po.Scanner(*SC_ARGS)
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


@pytest.mark.parametrize("projector,tof,rays,psf", [
    ("S", None, 1, False), ("S", (214.0, 5), 1, False), ("S", (214.0, 5), 4, False),
    ("DD", None, 1, False), ("DD", (214.0, 5), 1, True)])
def test_operator_projector_b200_through_the_reference_operator(projector, tof,
                                                                rays, psf,
                                                                tmp_path):
    po.ref_set_b200_precision(0)
    d1, d2 = random_events(15000, 60)
    rng = np.random.default_rng(61)
    tv = rng.normal(0, 250, len(d1)).astype(np.float32) if tof else None
    img = rng.uniform(0.2, 1.5, (1, IP_ARGS[2], IP_ARGS[1], IP_ARGS[0])).astype(np.float32)
    y = rng.uniform(0.1, 1.0, len(d1)).astype(np.float32)
    csv = None
    table = None
    if psf:
        table = gaussian_psf()
        csv = str(tmp_path / "psf.csv")
        yrt.write_psf_csv(csv, *table)
    osc, oip = po.Scanner(*SC_ARGS), po.ImageParams(*IP_ARGS)
    kw = dict(projector=projector, num_rays=rays,
              tof_fwhm_ps=tof[0] if tof else 0.0, tof_n_std=tof[1] if tof else 0,
              threads=8)
    bf = po.ref_project_lm(osc, oip, d1, d2, tof=tv, image=img, psf_csv=csv,
                           gpu="b200", **kw)
    bb = po.ref_project_lm(osc, oip, d1, d2, tof=tv, values=y, fwd=False,
                           psf_csv=csv, gpu="b200", **kw)
    rf = po.ref_project_lm(osc, oip, d1, d2, tof=tv, image=img, psf_csv=csv,
                           gpu=True, **kw)
    rb = po.ref_project_lm(osc, oip, d1, d2, tof=tv, values=y, fwd=False,
                           psf_csv=csv, gpu=True, **kw)
    assert rel_l2(bf, rf) < 1e-5
    assert rel_l2(bb, rb) < 1e-5
    # libyrtb's own projector on the detector pairs: same forward bits.
    sc = yrt.Scanner("t", *SC_ARGS)
    pp = yrt.ProjectorParams(sc)
    pp.setProjector(projector)
    pp.numRays = rays
    pp.precision = L.YRTB_MIRROR
    if tof:
        pp.addTOF(*tof)
    if psf:
        pp.setProjPsf(*table)
    p = yrt.DeviceProjector(sc, yrt.ImageParams(*IP_ARGS), pp)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    own = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    assert np.array_equal(own.view(np.uint32), bf.view(np.uint32))


def _c1(n, seed, tof):
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ev = S.generate_events(sc, n, seed, tof_fwhm_ps=214.0 if tof else None)
    return sc, ev.numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_reference_osem_driver_on_libyrtb_listmode(precision):
    # OSEM::reconstruct of the reference, list mode with TOF, a sensitivity
    # histogram, an attenuation image and per-event randoms: OSEM_GPU_B200
    # against OSEM_GPU on the same inputs, and against libyrtb's own driver.
    from pyyrtpet_b200 import synthetic as S
    sc, e = _c1(50000, 62, True)
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    eff = S.crystal_efficiencies(sc, 63).numpy()
    h = po.ref_histo3d_crystal_product(osc, eff)
    mu = S.Phantom(cyl_half_length=32).mu_image(ip).numpy()
    rnd = np.random.default_rng(64).uniform(0, 0.01, len(e["d1"])).astype(np.float32)
    sens, _ = po.ref_sensitivity(osc, oip, listmode=True, sens_histo=h,
                                 att_params=oip, att_image=mu, gpu=True)
    kw = dict(tof=e["tof"], randoms=rnd, sens_histo=h, att_params=oip,
              att_image=mu, iterations=2, subsets=3, tof_fwhm_ps=214.0,
              tof_n_std=5)
    po.ref_set_b200_precision(precision)
    img_b, _ = po.ref_osem_listmode(osc, oip, sens[0], e["d1"], e["d2"],
                                    gpu="b200", **kw)
    img_r, _ = po.ref_osem_listmode(osc, oip, sens[0], e["d1"], e["d2"],
                                    gpu=True, **kw)
    assert np.abs(img_b).sum() > 0
    if precision == 0:
        assert rel_l2(img_b, img_r) < 1e-4
    # libyrtb's own driver (yrtb_osem_listmode) on the same corrections.
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = precision
    p = yrt.DeviceProjector(sc, ip, pp)
    ev = yrt.DeviceEvents.from_arrays(e["d1"], e["d2"], tof=e["tof"],
                                      additive=rnd)
    ev.sens = p.gather_crystal_product(torch.from_numpy(eff).cuda(), ev)
    ev.att = p.attenuation_factors(torch.from_numpy(mu).cuda().reshape(-1), ip, ev)
    import ctypes
    from pyyrtpet_b200.core import _stream
    J = ip.numVoxels
    x = torch.empty(J, device="cuda")
    work = torch.empty(2 * J, device="cuda")
    s_d = torch.from_numpy(sens[0]).cuda().reshape(-1).contiguous()
    prm = L.yrtb_osem_params(2, 3, 1.0, 1e-35, 1.19209e-07, 0, 0, None, None)
    L.check(L.lib().yrtb_osem_listmode(p.h, ctypes.byref(ev.c()), s_d.data_ptr(),
                                       x.data_ptr(), work.data_ptr(),
                                       ctypes.byref(prm), _stream()))
    own = x.cpu().numpy()
    assert rel_l2(img_b, own) < 1e-4


def test_reference_osem_driver_on_libyrtb_histogram_dd_psf(tmp_path):
    # Histogram data (a MEASUREMENT property per bin) with distance-driven
    # projection and a projection-space PSF.
    sc, e = _c1(150000, 65, False)
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    hist, bad = po.lm_to_histo3d(osc, e["d1"], e["d2"])
    assert bad == 0
    csv = str(tmp_path / "psf.csv")
    yrt.write_psf_csv(csv, *gaussian_psf())
    sens, _ = po.ref_sensitivity(osc, oip, projector="DD", subsets=3,
                                 listmode=False, psf_csv=csv, gpu=True)
    po.ref_set_b200_precision(0)
    img_b, _ = po.ref_osem_histo3d(osc, oip, sens, hist, psf_csv=csv,
                                   projector="DD", iterations=1, subsets=3,
                                   gpu="b200")
    img_r, _ = po.ref_osem_histo3d(osc, oip, sens, hist, psf_csv=csv,
                                   projector="DD", iterations=1, subsets=3,
                                   gpu=True)
    assert np.abs(img_b).sum() > 0
    assert rel_l2(img_b, img_r) < 1e-4


def test_reference_osem_driver_on_libyrtb_dynamic_frames():
    # DynamicFraming (3 frames): the rows carry DYNAMIC_FRAME and the image
    # update runs per frame against the 3D sensitivity image.
    sc, e = _c1(60000, 66, True)
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128, nt=3)
    n = len(e["d1"])
    ts = np.sort(np.random.default_rng(67).integers(0, 3000, n)).astype(np.uint32)
    frame_ts = np.array([0, 1000, 2000, 3000], np.uint32)
    sens, _ = po.ref_sensitivity(osc, po.ImageParams(32, 32, 16, 256, 256, 128),
                                 listmode=True, gpu=True)
    kw = dict(frame_ts=frame_ts, tof=e["tof"], iterations=1, subsets=2,
              tof_fwhm_ps=214.0, tof_n_std=5)
    po.ref_set_b200_precision(0)
    img_b, _ = po.ref_osem_listmode_dynamic(osc, oip, sens[0], e["d1"], e["d2"],
                                            ts, gpu="b200", **kw)
    img_r, _ = po.ref_osem_listmode_dynamic(osc, oip, sens[0], e["d1"], e["d2"],
                                            ts, gpu=True, **kw)
    assert img_b.shape == (3, 16, 32, 32)
    assert rel_l2(img_b, img_r) < 1e-4
