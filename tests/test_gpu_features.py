"""Dynamic / motion OSEM against the reference, the differentiable projector
(torch.autograd), and the compensated precision mode.

Tolerances: rel-L2 1e-4 per reconstructed image against the reference;
gradients within 1e-4 relative of FP64 central differences (h = 2^-10) and of
the reference CPU back projector; adjoint identity to 1e-6.
"""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L
from pyyrtpet_b200 import synthetic as S
from pyyrtpet_b200.autograd import SiddonProjectFn, poisson_nll, poisson_nll_fused

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not po.ref_available(),
                               reason="reference library not built")
C1 = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@needs_ref
def test_dynamic_frames_and_motion_osem_vs_reference():
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    evs = S.generate_events(sc, 60000, 41, tof_fwhm_ps=214.0)
    e = evs.numpy()
    n = len(e["d1"])
    ts = np.sort(np.random.default_rng(42).integers(0, 10000, n)).astype(np.uint32)
    frame_ts = np.array([500, 3000, 6500, 9800], np.uint32)        # 3 frames
    motion_starts = np.array([2000, 7000], np.uint32)              # 2 motion frames
    motion = S.rigid_transforms(2, 43)
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e["tof"], timestamps=ts)
    lm.addDynamicFraming(frame_ts)
    lm.addLORMotion(motion_starts, motion)
    assert lm.getNumDynamicFrames() == 3
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 2
    osem.setListModeEnabled(True)
    osem.addTOF(214.0, 5)
    sens = osem.generateSensitivityImages()
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    assert img.shape == (3, 16, 32, 32)
    osc = po.Scanner(*C1)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128, nt=3)
    ref, _ = po.ref_osem_listmode_dynamic(
        osc, oip, sens[0].cpu().numpy(), e["d1"], e["d2"], ts,
        frame_ts=frame_ts, motion_starts=motion_starts, motion=motion,
        tof=e["tof"], iterations=2, subsets=2, tof_fwhm_ps=214.0, tof_n_std=5)
    assert rel_l2(img, ref) < 1e-4


def _c1_setup(n, seed, nx=32, nz=16):
    sc = S.scanner_c1()
    ip = yrt.ImageParams(nx, nx, nz, 256, 256, 128)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    proj = yrt.DeviceProjector(sc, ip, pp)
    evs = S.generate_events(sc, n, seed, tof_fwhm_ps=214.0)
    e = evs.numpy()
    ev = yrt.DeviceEvents.from_arrays(e["d1"], e["d2"], tof=e["tof"])
    return sc, ip, proj, ev, e


def test_autograd_gradient_vs_fp64_finite_differences():
    sc, ip, proj, ev, e = _c1_setup(20000, 51)
    rng = np.random.default_rng(52)
    # x0 in [0.5, 0.99) and h = 2^-10 keep x0 +/- h exact in float32, so
    # the FP64 differences see exactly the perturbation they divide by.
    x0 = rng.uniform(0.5, 0.99, ip.shape).astype(np.float32)
    sens = rng.uniform(0.5, 1.0, ip.shape).astype(np.float32)
    x = torch.from_numpy(x0).cuda().requires_grad_(True)
    loss = poisson_nll(x, proj, ev, torch.from_numpy(sens).cuda())
    loss.backward()
    g = x.grad.cpu().numpy().ravel()
    # FP64 loss from the oracle's FP64 forward projector.
    lut = po.scanner_lut(po.Scanner(*C1))
    lors, _ = po.lors_from_detpairs(lut, e["d1"], e["d2"])
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    pr = po.Proj(tof_fwhm_ps=214.0, tof_n_std=5)

    def loss64(xv):
        y = po.project(oip, pr, lors, image=xv.astype(np.float32), tof=e["tof"],
                       precision="f64")
        return float(np.sum(sens.astype(np.float64) * xv) - np.sum(np.log(y[y > 0])))

    # Voxels with a meaningful gradient (inside the FOV, crossed by events).
    cand = np.nonzero(np.abs(g) > 1e-2 * np.abs(g).max())[0]
    pick = rng.choice(cand, 64, replace=False)
    h = 2.0 ** -10
    base = x0.astype(np.float64).ravel()
    errs = []
    for j in pick:
        xp = base.copy()
        xm = base.copy()
        xp[j] += h
        xm[j] -= h
        fd = (loss64(xp.reshape(ip.shape)) - loss64(xm.reshape(ip.shape))) / (2 * h)
        errs.append(abs(fd - g[j]) / max(abs(fd), 1e-12))
    assert np.median(errs) < 1e-5
    assert max(errs) < 1e-4


@needs_ref
def test_autograd_gradient_vs_reference_backprojector():
    sc, ip, proj, ev, e = _c1_setup(30000, 53)
    rng = np.random.default_rng(54)
    x0 = rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)
    sens = np.ones(ip.shape, np.float32)
    x = torch.from_numpy(x0).cuda().requires_grad_(True)
    y = SiddonProjectFn.apply(x, proj, ev)
    loss = (torch.from_numpy(sens).cuda() * x).sum() - torch.log(y.clamp_min(1e-12)).sum()
    loss.backward()
    yh = y.detach().cpu().numpy()
    w = np.where(yh > 1e-12, 1.0 / np.maximum(yh, 1e-12), 0.0).astype(np.float32)
    lut = po.scanner_lut(po.Scanner(*C1))
    lors, _ = po.lors_from_detpairs(lut, e["d1"], e["d2"])
    ref_bp = po.ref_siddon(po.Scanner(*C1), po.ImageParams(32, 32, 16, 256, 256, 128),
                           lors, values=w, tof=e["tof"], tof_fwhm_ps=214.0,
                           tof_n_std=5, forward=False)
    ref_grad = sens - ref_bp
    assert rel_l2(x.grad.cpu().numpy(), ref_grad) < 1e-4


def test_autograd_batched_and_adjoint():
    sc, ip, proj, ev, e = _c1_setup(20000, 55)
    rng = np.random.default_rng(57)
    xb = torch.from_numpy(rng.uniform(0, 1, (2,) + ip.shape).astype(np.float32)).cuda()
    xb.requires_grad_(True)
    # One event set per phantom (different counts -> list of projections).
    ys = SiddonProjectFn.apply(xb, proj, [ev, ev])
    y = SiddonProjectFn.apply(xb, proj, ev)
    assert torch.equal(ys, y)
    assert y.shape == (2, ev.count)
    gy = torch.from_numpy(rng.uniform(0, 1, (2, ev.count)).astype(np.float32)).cuda()
    (y * gy).sum().backward()
    for b in range(2):
        lhs = float((y[b].detach().double() * gy[b].double()).sum())
        rhs = float((xb[b].detach().double() * xb.grad[b].double()).sum())
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    # torch.autograd.gradcheck-style check of linearity: A(a x) = a A(x).
    y2 = SiddonProjectFn.apply(2.0 * xb.detach(), proj, ev)
    assert rel_l2(y2.cpu().numpy(), 2.0 * y.detach().cpu().numpy()) < 1e-6


@pytest.mark.parametrize("precision", [L.YRTB_MIRROR, L.YRTB_COMPENSATED])
def test_fused_poisson_nll_matches_composed(precision):
    # One fused pass per event set (yrtb_em_step_model) gives the same loss
    # as forward projection + torch reductions (identical forward sums, FP64
    # sums) and the same gradient as autograd through the adjoint kernel, up
    # to the order of the FP32 atomic sums (1e-6 relative L2).
    sc, ip, _, ev, e = _c1_setup(30000, 71)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = precision
    proj = yrt.DeviceProjector(sc, ip, pp)
    e2 = S.generate_events(sc, 30000, 73, tof_fwhm_ps=214.0).numpy()
    ev2 = yrt.DeviceEvents.from_arrays(e2["d1"], e2["d2"], tof=e2["tof"])
    rng = np.random.default_rng(72)
    x0 = torch.from_numpy(rng.uniform(0.0, 1.0, (2,) + ip.shape).astype(np.float32)).cuda()
    sens = torch.from_numpy(rng.uniform(0.5, 1.0, ip.shape).astype(np.float32)).cuda()
    for x_init, evs in ((x0[0], ev), (x0, [ev, ev2])):
        xa = x_init.clone().requires_grad_(True)
        xb = x_init.clone().requires_grad_(True)
        la = poisson_nll(xa, proj, evs, sens)
        lb = poisson_nll_fused(xb, proj, evs, sens)
        assert torch.equal(la, lb)
        w = torch.arange(1, la.numel() + 1, dtype=la.dtype, device=la.device).reshape(la.shape)
        (w * la).sum().backward()
        (w * lb).sum().backward()
        assert rel_l2(xb.grad.cpu().numpy(), xa.grad.cpu().numpy()) < 1e-6


def test_compensated_mode_error_vs_fp64():
    sc = S.scanner_c1()
    ip = yrt.ImageParams(64, 64, 32, 256, 256, 128)
    evs = S.generate_events(sc, 40000, 61, tof_fwhm_ps=214.0)
    e = evs.numpy()
    rng = np.random.default_rng(62)
    img = rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)
    outs = {}
    for prec in (L.YRTB_MIRROR, L.YRTB_COMPENSATED):
        pp = yrt.ProjectorParams(sc)
        pp.addTOF(214.0, 5)
        pp.precision = prec
        p = yrt.DeviceProjector(sc, ip, pp)
        ev = yrt.DeviceEvents.from_arrays(e["d1"], e["d2"], tof=e["tof"])
        outs[prec] = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    lut = po.scanner_lut(po.Scanner(*C1))
    lors, _ = po.lors_from_detpairs(lut, e["d1"], e["d2"])
    oip = po.ImageParams(64, 64, 32, 256, 256, 128)
    pr = po.Proj(tof_fwhm_ps=214.0, tof_n_std=5)
    f32 = po.project(oip, pr, lors, image=img, tof=e["tof"])
    f64 = po.project(oip, pr, lors, image=img, tof=e["tof"], precision="f64")
    # Mirror mode reproduces the reference's FP32 arithmetic (only the TOF
    # exponential differs, <= 2 ulp) ...
    assert rel_l2(outs[L.YRTB_MIRROR], f32) < 1e-6
    # ... including its error on rays that run within float rounding of a
    # voxel boundary (LORs between crystals on the x or y axis through the
    # centre of this 4 mm grid), where FP32 puts the entry voxel on the other
    # side of the plane: the reference's own error vs FP64 here is ~1e-3.
    err_ref = rel_l2(f32, f64)
    # Compensated mode takes the entry set-up in FP64 and meets the budget.
    err_c = rel_l2(outs[L.YRTB_COMPENSATED], f64)
    assert err_c < 1e-5
    assert err_c < err_ref


@pytest.mark.parametrize("tof,randoms", [(False, False), (True, False), (True, True)])
def test_listmode_file_unpacked_on_gpu(tmp_path, tof, randoms):
    sc = S.scanner_c1()
    rng = np.random.default_rng(81)
    n = 100003
    lm = yrt.ListModeLUT(sc, tof, randoms)
    lm.allocate(n)
    lm.timestamps[:] = np.sort(rng.integers(0, 1 << 30, n))
    lm.d1[:] = rng.integers(0, sc.getNumDets(), n)
    lm.d2[:] = rng.integers(0, sc.getNumDets(), n)
    if tof:
        lm.tof[:] = rng.normal(0, 300, n)
    if randoms:
        lm.randoms[:] = rng.uniform(0, 1, n)
    f = str(tmp_path / "events.lmDat")
    lm.writeToFile(f)
    got = yrt.ListModeLUT(sc, tof, randoms).readFromFile(f, device=True)
    assert np.array_equal(got.d1, lm.d1) and np.array_equal(got.d2, lm.d2)
    assert np.array_equal(got.timestamps, lm.timestamps)
    if tof:
        assert np.array_equal(got.tof.view(np.uint32), lm.tof.view(np.uint32))
        assert torch.equal(got.device_events().tof.cpu(), torch.from_numpy(lm.tof))
    if randoms:
        assert np.array_equal(got.randoms.view(np.uint32), lm.randoms.view(np.uint32))
    if po.ref_available():
        ts, a, b, tv, rv = po.ref_read_listmode(po.Scanner(*C1), f, tof, randoms, n)
        assert np.array_equal(a, got.d1) and np.array_equal(b, got.d2)
        assert np.array_equal(ts, got.timestamps)
        if tof:
            assert np.array_equal(tv.view(np.uint32), got.tof.view(np.uint32))
    # An invalid detector id is reported with the event index, as the
    # reference reader does.
    raw = np.fromfile(f, np.uint32).reshape(n, -1)
    raw[777, 2] = sc.getNumDets() + 5
    raw.tofile(f)
    with pytest.raises(yrt.YrtbError, match="list-mode event 777"):
        yrt.ListModeLUT(sc, tof, randoms).readFromFile(f, device=True)


def test_distributed_osem_driver_matches_c_driver_on_one_rank():
    """pyyrtpet_b200.distributed.osem_listmode (the sharded driver, run here
    without a process group) against yrtb_osem_listmode on the same ordered
    events: same steps, so the images agree to float summation order."""
    import ctypes
    from pyyrtpet_b200 import synthetic as S
    from pyyrtpet_b200.core import _stream
    from pyyrtpet_b200.distributed import osem_listmode
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = L.YRTB_COMPENSATED
    proj = yrt.DeviceProjector(sc, ip, pp)
    e = S.generate_events(sc, 40000, 77, tof_fwhm_ps=214.0, device="cuda")
    ev = yrt.DeviceEvents.from_arrays(e.d1.to(torch.int32), e.d2.to(torch.int32),
                                      tof=e.tof)
    ev, offs = proj.order_events(ev, 4)
    sens = torch.zeros(ip.numVoxels, device="cuda")
    sp = yrt.DeviceProjector(sc, ip, yrt.ProjectorParams(sc))
    sp.sensitivity_histo3d(sens, 1, 0)
    a = torch.empty(ip.numVoxels, device="cuda")
    osem_listmode(proj, ev, offs, sens, a, 2, 4)
    b = torch.empty(ip.numVoxels, device="cuda")
    work = torch.empty(2 * ip.numVoxels, device="cuda")
    p = L.yrtb_osem_params(2, 4, 1.0, 1e-35, 1.19209e-07, 0, 0, None, offs.ctypes.data)
    L.check(L.lib().yrtb_osem_listmode(proj.h, ctypes.byref(ev.c()), sens.data_ptr(),
                                       b.data_ptr(), work.data_ptr(), ctypes.byref(p),
                                       _stream()))
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-6
