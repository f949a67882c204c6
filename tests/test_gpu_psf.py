"""Image-space PSF on the device (yrtb_psf_*, OperatorPsfDevice) and OSEM
with an image-space PSF, against the reference OperatorPsf and OSEM_CPU
(src/operators/OperatorPsf.cpp:288-375, src/recon/OSEM_CPU.cpp:150-230)."""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt

pytestmark = pytest.mark.gpu

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
needs_ref = pytest.mark.skipif(not po.ref_available(),
                               reason="reference library not built")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("adjoint", [False, True])
@pytest.mark.parametrize("shape,sizes", [((2, 12, 16, 20), (5, 7, 3)),
                                         ((1, 9, 33, 31), (1, 9, 17)),
                                         ((1, 5, 4, 3), (5, 7, 9)),
                                         ((3, 7, 10, 36), (15, 11, 13)),
                                         ((1, 6, 9, 8), (7, 3, 5)),
                                         ((1, 4, 8, 24), (19, 1, 3))])
def test_psf_apply_matches_oracle_bitexact(adjoint, shape, sizes):
    """FP32 sums in tap order with circular borders: bit-identical to the
    oracle's restatement (itself pinned to the reference operator)."""
    nt, nz, ny, nx = shape
    rng = np.random.default_rng(71 + nx)
    img = rng.random(shape, dtype=np.float32)
    ks = [rng.random(n).astype(np.float32) for n in sizes]
    oip = po.ImageParams(nx, ny, nz, 2.0 * nx, 2.0 * ny, 2.0 * nz, nt=nt)
    ip = yrt.ImageParams(nx, ny, nz, 2.0 * nx, 2.0 * ny, 2.0 * nz, nt=nt)
    expect = po.psf_convolve(oip, img, *ks, adjoint=adjoint)
    psf = yrt.OperatorPsfDevice(*ks)
    d_in = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_in)
    (psf.applyAH if adjoint else psf.applyA)(d_in, d_out, ip)
    torch.cuda.synchronize()
    assert np.array_equal(bits(d_out.cpu().numpy()), bits(expect))


@needs_ref
@pytest.mark.parametrize("adjoint", [False, True])
def test_psf_apply_matches_reference_operator(adjoint):
    rng = np.random.default_rng(72)
    img = rng.random((2, 12, 16, 20), dtype=np.float32)
    ks = [rng.random(n).astype(np.float32) for n in (5, 7, 3)]
    oip = po.ImageParams(20, 16, 12, 40, 32, 24, nt=2)
    ref = po.ref_psf_convolve(oip, img, *ks, adjoint=adjoint)
    psf = yrt.OperatorPsfDevice(*ks)
    d_in = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_in)
    (psf.applyAH if adjoint else psf.applyA)(d_in, d_out)
    assert np.array_equal(bits(d_out.cpu().numpy()), bits(ref))


def test_psf_adjoint_identity():
    """<A x, y> = <x, A^H y> within float rounding."""
    rng = np.random.default_rng(73)
    shape = (1, 24, 40, 36)
    x = torch.from_numpy(rng.random(shape, dtype=np.float32)).cuda()
    y = torch.from_numpy(rng.random(shape, dtype=np.float32)).cuda()
    psf = yrt.OperatorPsfDevice.createGaussianFromFWHM(4.0, 4.0, 5.0, 2.0, 2.0, 2.5)
    ax = torch.empty_like(x)
    ahy = torch.empty_like(y)
    psf.applyA(x, ax)
    psf.applyAH(y, ahy)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * ahy.double()).sum())
    assert abs(lhs - rhs) / abs(rhs) < 1e-6


def test_psf_gaussian_preserves_total_and_symmetry():
    """A normalised symmetric kernel keeps the image total (circular borders)
    and makes applyA = applyAH."""
    rng = np.random.default_rng(74)
    x = torch.from_numpy(rng.random((1, 16, 32, 32), dtype=np.float32)).cuda()
    psf = yrt.OperatorPsfDevice.createGaussianFromSigma(1.5, 1.5, 2.0, 2.0, 2.0, 2.0)
    a = torch.empty_like(x)
    ah = torch.empty_like(x)
    psf.applyA(x, a)
    psf.applyAH(x, ah)
    assert abs(float(a.double().sum()) - float(x.double().sum())) < 1e-4 * float(x.double().sum())
    assert torch.equal(a, ah)


def test_psf_argument_errors():
    with pytest.raises(RuntimeError):
        yrt.OperatorPsfDevice(np.ones(4, np.float32), np.ones(3, np.float32),
                              np.ones(3, np.float32))
    psf = yrt.OperatorPsfDevice(np.ones(9, np.float32), np.ones(3, np.float32),
                                np.ones(3, np.float32))
    x = torch.ones((1, 4, 4, 4), device="cuda")
    with pytest.raises(RuntimeError):  # half-width 4 >= nx 4
        psf.applyA(x, torch.empty_like(x))
    with pytest.raises(RuntimeError):
        psf.applyA(x, x)


def _c1_events(n, seed, tof=False):
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128)
    ev = S.generate_events(sc, n, seed, tof_fwhm_ps=214.0 if tof else None)
    return sc, ip, ev.numpy()


def _psf_csv(tmp_path):
    kx = yrt.OperatorPsfDevice.createGaussianKernel1D(4.0 / 2.35482, 8.0, 5)
    kz = yrt.OperatorPsfDevice.createGaussianKernel1D(5.0 / 2.35482, 8.0, 3)
    fname = str(tmp_path / "image_psf.csv")
    yrt.write_image_psf_csv(fname, kx, kx, kz)
    return fname


@needs_ref
@pytest.mark.parametrize("tof", [False, True])
def test_listmode_osem_with_image_psf_vs_reference(tmp_path, tof):
    sc, ip, e = _c1_events(60000, 81, tof)
    csv = _psf_csv(tmp_path)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 3
    osem.setListModeEnabled(True)
    if tof:
        osem.addTOF(214.0, 5)
    osem.addImagePSF(csv)
    assert osem.hasImagePSF()
    sens = osem.generateSensitivityImages()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    rs, _ = po.ref_sensitivity(osc, oip, listmode=True, image_psf_csv=csv)
    assert rel_l2(sens[0].cpu().numpy(), rs[0]) < 1e-5
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e.get("tof"))
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"],
                                  tof=e.get("tof"), iterations=2, subsets=3,
                                  tof_fwhm_ps=214.0 if tof else 0.0,
                                  tof_n_std=5 if tof else 0, image_psf_csv=csv)
    assert rel_l2(img, ref) < 1e-4


@needs_ref
def test_histogram_osem_with_image_psf_vs_reference(tmp_path):
    sc, ip, e = _c1_events(200000, 82)
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"])
    hist = yrt.convertToHistogram3D(lm)
    csv = _psf_csv(tmp_path)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 1
    osem.num_OSEM_subsets = 4
    osem.addImagePSF(csv)
    osem.setDataInput(hist)
    sens = osem.generateSensitivityImages()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    rs, _ = po.ref_sensitivity(osc, oip, subsets=4, listmode=False,
                               image_psf_csv=csv)
    for s in range(4):
        assert rel_l2(sens[s].cpu().numpy(), rs[s]) < 1e-5
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_histo3d(osc, oip, rs, hist.data, iterations=1,
                                 subsets=4, image_psf_csv=csv)
    assert rel_l2(img, ref) < 1e-4


def test_gaussian_image_psf_equals_csv_psf(tmp_path):
    """addUniformGaussianImagePSFFromFWHM builds the same kernels as the
    CSV it would be written to."""
    sc, ip, e = _c1_events(20000, 83)
    outs, kernels = [], []
    for how in ("gauss", "csv"):
        osem = yrt.createOSEM(sc)
        osem.setImageParams(ip)
        osem.num_MLEM_iterations = 1
        osem.num_OSEM_subsets = 2
        osem.setListModeEnabled(True)
        if how == "gauss":
            osem.addUniformGaussianImagePSFFromFWHM(6.0, 6.0, 8.0)
        else:
            p = yrt.OperatorPsfDevice.createGaussianFromFWHM(6.0, 6.0, 8.0, ip.vx, ip.vy, ip.vz)
            fname = str(tmp_path / "g.csv")
            yrt.write_image_psf_csv(fname, p.getKernelX(), p.getKernelY(), p.getKernelZ())
            osem.addImagePSF(fname)
        osem.generateSensitivityImages()
        lm = yrt.ListModeLUT(sc)
        lm.bind(e["d1"], e["d2"])
        osem.setDataInput(lm)
        outs.append(osem.reconstruct().cpu().numpy())
        kernels.append([osem.imagePsf.getKernelX(), osem.imagePsf.getKernelY(),
                        osem.imagePsf.getKernelZ()])
    for a, b in zip(*kernels):
        assert np.array_equal(bits(a), bits(b))
    # The back projection's float atomics sum in arrival order.
    assert rel_l2(outs[0], outs[1]) < 1e-5


def test_image_psf_graph_and_plain_agree(tmp_path):
    sc, ip, e = _c1_events(30000, 84, tof=True)
    csv = _psf_csv(tmp_path)
    outs = []
    for graphs in (False, True):
        osem = yrt.createOSEM(sc)
        osem.setImageParams(ip)
        osem.num_MLEM_iterations = 2
        osem.num_OSEM_subsets = 2
        osem.setListModeEnabled(True)
        osem.addTOF(214.0, 5)
        osem.addImagePSF(csv)
        osem.useGraphs = graphs
        osem.generateSensitivityImages()
        lm = yrt.ListModeLUT(sc)
        lm.bind(e["d1"], e["d2"], tof=e["tof"])
        osem.setDataInput(lm)
        outs.append(osem.reconstruct().cpu().numpy())
    # Same launches in both; only the arrival order of float atomics differs.
    assert rel_l2(outs[1], outs[0]) < 1e-5


# ------------------------------------------- spatially variant image PSF --
def _varpsf_csv(path, two_gaussian, seed):
    """LUT of the reference's VarPSF unit test: 5 x 5 x 5 kernels over range
    200 mm, gap 50 mm, 4 sigmas, sigmas switching at 100 mm
    (unit_tests/operators/test_PSF.cpp:290-360)."""
    rng = np.random.default_rng(seed)
    s1lo, s1hi = rng.uniform(0.5, 1.0, 3), rng.uniform(1.1, 1.5, 3)
    s2lo, s2hi = rng.uniform(1.6, 2.0, 3), rng.uniform(2.1, 2.5, 3)
    w2 = rng.uniform(0.2, 0.6)
    vals = [5.1, 54.9, 105.3, 155.1, 205.5]
    rows = []
    for z in vals:
        for y in vals:
            for x in vals:
                pos = (x, y, z)
                s1 = [s1hi[a] if pos[a] > 100 else s1lo[a] for a in range(3)]
                s2 = [s2hi[a] if pos[a] > 100 else s2lo[a] for a in range(3)]
                rows.append(s1 + s2 + [w2] if two_gaussian else s1)
    with open(path, "w") as f:
        f.write("200,200,200\n50,50,50\n4,4,4\n")
        for r in rows:
            f.write(",".join(f"{float(v):.9g}" for v in r) + "\n")
    return path


@needs_ref
@pytest.mark.parametrize("two_gaussian", [False, True])
def test_varpsf_vs_reference_operator(tmp_path, two_gaussian):
    ip = yrt.ImageParams(100, 100, 51, 400.0, 401.0, 421.0)
    oip = po.ImageParams(100, 100, 51, 400.0, 401.0, 421.0)
    csv = _varpsf_csv(str(tmp_path / "v.csv"), two_gaussian, 95)
    rng = np.random.default_rng(96)
    img = rng.random((51, 100, 100), dtype=np.float32)
    op = yrt.OperatorVarPsfDevice(csv, ip)
    d_in = torch.from_numpy(img).cuda()
    fwd = op.applyA(d_in, torch.empty_like(d_in)).cpu().numpy()
    ref = po.ref_varpsf_apply(oip, csv, img)
    assert np.array_equal(bits(fwd), bits(ref))
    adj = op.applyAH(d_in, torch.empty_like(d_in)).cpu().numpy()
    ref_adj = po.ref_varpsf_apply(oip, csv, img, adjoint=True)
    assert rel_l2(adj, ref_adj) < 1e-6
    y = torch.from_numpy(rng.random((51, 100, 100), dtype=np.float32)).cuda()
    lhs = float((torch.from_numpy(fwd).cuda().double() * y.double()).sum())
    rhs = float((d_in.double() * op.applyAH(y, torch.empty_like(y)).double()).sum())
    assert abs(lhs - rhs) / abs(rhs) < 1e-6


@needs_ref
def test_listmode_osem_with_variant_psf_vs_reference(tmp_path):
    sc, ip, e = _c1_events(60000, 97)
    rng = np.random.default_rng(98)
    csv = str(tmp_path / "v.csv")
    with open(csv, "w") as f:
        f.write("60,60,30\n30,30,30\n3,3,3\n")
        for _ in range(3 * 3 * 2):
            f.write(",".join(f"{v:.6g}" for v in rng.uniform(6.0, 12.0, 3)) + "\n")
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 2
    osem.setListModeEnabled(True)
    osem.addImagePSF(csv, "VARIANT")
    sens = osem.generateSensitivityImages()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128)
    rs, _ = po.ref_sensitivity(osc, oip, listmode=True, image_psf_csv=csv,
                               image_psf_variant=True)
    assert rel_l2(sens[0].cpu().numpy(), rs[0]) < 1e-5
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"])
    osem.setDataInput(lm)
    img = osem.reconstruct().cpu().numpy()
    ref, _ = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"], iterations=2,
                                  subsets=2, image_psf_csv=csv, image_psf_variant=True)
    assert rel_l2(img, ref) < 1e-4
