"""The CUDA path against the reference's own CUDA path on the same GPU.

The second oracle: YRT-PET 2.0.7 compiled with BUILD_CUDA for sm_100a
(oracle/ref_cuda.mk -> oracle/_ref_cuda/).  Its list-mode projections run
OperatorProjectorDevice with projectSiddon_kernel / projectDD_kernel
(include/yrt-pet/operators/SiddonKernels.cuh:502-574,
include/yrt-pet/operators/DDKernels.cuh:398-463) through util::forwProject /
util::backProject (src/utils/ReconstructionUtils.cpp:948-1061), and its OSEM
runs OSEM_GPU with computeEMUpdateImage_kernel (src/recon/OSEM_GPU.cu:1159-1341).

Tolerances (stated per test): relative L2 <= 1e-5 per projection vector and
<= 1e-4 per image.  The reference's device code is compiled with nvcc's
default FMA contraction, so it is not bit-identical to its own CPU projector;
the libyrtb mirror mode is (non-TOF), so both are compared at the stated
tolerance rather than bit for bit.

Multi-ray: the reference device path draws each event's offsets with
curand_init(13, event index in the batch, 0) (SiddonKernels.cuh:27-84).  A
different stream moves every extra ray by up to half a crystal, which changes
single projections by tens of percent; the per-event bound below therefore
pins the stream, not only the average.
"""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not po.ref_gpu_available(),
                                 reason="reference CUDA library not built")]

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
# An image with an offset, as the reference's own GPU-vs-CPU test uses
# (unit_tests/operators/test_Siddon_GPU.cu:28-35).
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


def make(projector="S", tof=None, num_rays=1, psf=None,
         precision=L.YRTB_MIRROR):
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*IP_ARGS)
    pp = yrt.ProjectorParams(sc)
    pp.setProjector(projector)
    pp.numRays = num_rays
    pp.precision = precision
    if tof:
        pp.addTOF(*tof)
    if psf is not None:
        pp.setProjPsf(*psf)
    return yrt.DeviceProjector(sc, ip, pp)


def gaussian_psf(fwhm=4.0, ks=0.5):
    sig = fwhm / 2.3548
    half = int(np.ceil(3 * sig / ks))
    x = (np.arange(2 * half + 1) - half) * ks
    k = np.exp(-0.5 * (x / sig) ** 2)
    k /= k.sum() * ks
    return 1e9, ks, k[None].astype(np.float32)


def ref_kw(projector="S", tof=None, num_rays=1):
    return dict(projector=projector, num_rays=num_rays,
                tof_fwhm_ps=tof[0] if tof else 0.0,
                tof_n_std=tof[1] if tof else 0, threads=8)


def ours_and_ref(projector, tof, num_rays, psf_csv, table, precision, n, seed):
    d1, d2 = random_events(n, seed)
    rng = np.random.default_rng(seed + 1)
    tv = rng.normal(0, 250, len(d1)).astype(np.float32) if tof else None
    img = rng.uniform(0.2, 1.5, (1, IP_ARGS[2], IP_ARGS[1], IP_ARGS[0])) \
             .astype(np.float32)
    y = rng.uniform(0.1, 1.0, len(d1)).astype(np.float32)
    p = make(projector, tof, num_rays, table, precision)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tv)
    fwd = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    bwd = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    osc, oip = po.Scanner(*SC_ARGS), po.ImageParams(*IP_ARGS)
    kw = ref_kw(projector, tof, num_rays)
    rfwd = po.ref_project_lm(osc, oip, d1, d2, tof=tv, image=img,
                             psf_csv=psf_csv, gpu=True, **kw)
    rbwd = po.ref_project_lm(osc, oip, d1, d2, tof=tv, values=y, fwd=False,
                             psf_csv=psf_csv, gpu=True, **kw)
    return fwd, bwd, rfwd, rbwd, (osc, oip, d1, d2, tv, img, y, kw)


@pytest.mark.parametrize("precision", [L.YRTB_MIRROR, L.YRTB_COMPENSATED])
@pytest.mark.parametrize("tof", [None, (214.0, 5)])
def test_siddon_vs_reference_gpu(tof, precision):
    fwd, bwd, rfwd, rbwd, ctx = ours_and_ref("S", tof, 1, None, None,
                                             precision, 20000, 40)
    assert rel_l2(fwd, rfwd) < 1e-5
    assert rel_l2(bwd, rbwd) < 1e-5
    # Context: the reference GPU path against the reference CPU path on the
    # same events agrees to the same tolerance.
    osc, oip, d1, d2, tv, img, y, kw = ctx
    cfwd = po.ref_project_lm(osc, oip, d1, d2, tof=tv, image=img, **kw)
    assert rel_l2(rfwd, cfwd) < 1e-5


@pytest.mark.parametrize("tof", [None, (214.0, 5)])
def test_multiray_stream_vs_reference_gpu(tof):
    fwd, bwd, rfwd, rbwd, _ = ours_and_ref("S", tof, 4, None, None,
                                           L.YRTB_MIRROR, 20000, 41)
    assert rel_l2(fwd, rfwd) < 1e-5
    assert rel_l2(bwd, rbwd) < 1e-5
    # Per event: every projection with a non-negligible value agrees to 1e-3
    # relative, which a different random stream could not meet.
    big = np.abs(rfwd) > 1e-3 * np.abs(rfwd).max()
    assert big.sum() > 1000
    rel = np.abs(fwd[big] - rfwd[big]) / np.abs(rfwd[big])
    assert rel.max() < 1e-3


@pytest.mark.parametrize("precision", [L.YRTB_MIRROR, L.YRTB_COMPENSATED])
@pytest.mark.parametrize("tof,psf", [(None, False), ((214.0, 5), False),
                                     (None, True), ((214.0, 5), True)])
def test_dd_vs_reference_gpu(tof, psf, precision, tmp_path):
    table = gaussian_psf() if psf else None
    csv = None
    if psf:
        csv = str(tmp_path / "psf.csv")
        yrt.write_psf_csv(csv, *table)
    fwd, bwd, rfwd, rbwd, _ = ours_and_ref("DD", tof, 1, csv, table,
                                           precision, 12000, 42)
    assert rel_l2(fwd, rfwd) < 1e-5
    assert rel_l2(bwd, rbwd) < 1e-5


def _c1_problem(n, seed, tof):
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    ev = S.generate_events(sc, n, seed, tof_fwhm_ps=214.0 if tof else None)
    return sc, ip, ev


@pytest.mark.parametrize("tof", [False, True])
def test_sensitivity_and_listmode_osem_vs_reference_gpu(tof):
    sc, ip, evs = _c1_problem(60000, 43, tof)
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
    rs, _ = po.ref_sensitivity(osc, oip, listmode=True, gpu=True)
    assert rel_l2(sens[0].cpu().numpy(), rs[0]) < 1e-5
    e = evs.numpy()
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e.get("tof"))
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"],
                                  tof=e.get("tof"), iterations=2, subsets=3,
                                  tof_fwhm_ps=214.0 if tof else 0.0,
                                  tof_n_std=5 if tof else 0, gpu=True)
    assert rel_l2(img, ref) < 1e-4


def test_listmode_osem_with_corrections_vs_reference_gpu():
    from pyyrtpet_b200 import synthetic as S
    sc, ip, evs = _c1_problem(40000, 44, True)
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    h = yrt.Histogram3D(sc)
    eff = S.crystal_efficiencies(sc, 20).numpy()
    a, b = yrt.histo3d_detpairs(sc, np.arange(h.count(), dtype=np.uint64))
    h.data = (eff[a] * eff[b]).astype(np.float32)
    mu = S.Phantom(cyl_half_length=32).mu_image(ip).numpy()
    e = evs.numpy()
    rng = np.random.default_rng(45)
    randoms = rng.uniform(0.0, 0.01, len(e["d1"])).astype(np.float32)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 2
    osem.setListModeEnabled(True)
    osem.addTOF(214.0, 5)
    osem.setSensitivityHistogram(h)
    osem.setAttenuationImage(mu, ip)
    sens = osem.generateSensitivityImages()
    rs, _ = po.ref_sensitivity(osc, oip, listmode=True, sens_histo=h.data,
                               att_params=oip, att_image=mu, gpu=True)
    assert rel_l2(sens[0].cpu().numpy(), rs[0]) < 1e-5
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e["tof"], randoms=randoms)
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"],
                                  tof=e["tof"], randoms=randoms,
                                  sens_histo=h.data, att_params=oip,
                                  att_image=mu, iterations=2, subsets=2,
                                  tof_fwhm_ps=214.0, tof_n_std=5, gpu=True)
    assert rel_l2(img, ref) < 1e-4


def test_histogram_osem_dd_psf_vs_reference_gpu(tmp_path):
    sc, ip, evs = _c1_problem(200000, 46, False)
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
                               listmode=False, psf_csv=csv, gpu=True)
    for s in range(4):
        assert rel_l2(sens[s].cpu().numpy(), rs[s]) < 1e-5
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_histo3d(osc, oip, rs, hist.data, psf_csv=csv,
                                 projector="DD", iterations=1, subsets=4,
                                 gpu=True)
    assert rel_l2(img, ref) < 1e-4
