"""Pins the CPU oracle to the reference: its unit-test known answers, the
committed golden fixture made from the reference library, and (when the
reference library was built here) the reference itself on random inputs."""
import math
import os

import numpy as np
import pytest

import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "ref_small.npz"))

SC = po.Scanner(64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)
IP = po.ImageParams(32, 32, 16, 128, 128, 64)
needs_ref = pytest.mark.skipif(not po.ref_available(),
                               reason="reference library not built here")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


# --------------------------------------------------------- known answers --
def test_tof_weight_kat():
    # unit_tests/operators/test_TimeOfFlight.cpp:36-48
    p1 = np.array([-155.0, 118.75, 367.5], np.float32)
    p2 = np.array([155.0, 163.75, 373.5], np.float32)
    d = p2 - p1
    d_norm = np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))
    out = po.tof_f32(95.0, 3, d_norm, -408.0, np.float32(0.24) * d_norm,
                     np.float32(0.25) * d_norm)
    assert abs(out[0] - 0.000543244) < 1e-4


def test_tof_width_zero_full_range():
    # test_TimeOfFlight.cpp:21-34: width 0 -> alpha range [0, 1]
    out = po.tof_f32(0.0, 3, 1.5, -0.3, 0.1, 0.2)
    assert out[1] == 0.0 and out[2] == 1.0


@pytest.mark.parametrize("args,expected", [
    ((1.1, 4.1, 2.1, 3.1), 1.0), ((4, 1, 2, 3), 0.0), ((4.5, 2.3, 1.6, 3.2), 0.0),
    ((1.1, 1.2, 1.3, 1.4), 0.0), ((1.4, 1.3, 1.1, 1.2), 0.0),
    ((9.2, 10.9, 8.3, 10.0), 10.0 - 9.2), ((9.2, 9.9, 8.3, 10.0), 9.9 - 9.2)])
def test_dd_overlap_kats(args, expected):
    # unit_tests/operators/test_DD.cpp:24-32 (getOverlap = max(0, min - max))
    p0, p1, d0, d1 = (np.float32(v) for v in args)
    ov = max(np.float32(0), min(p1, d1) - max(p0, d0))
    assert ov == pytest.approx(expected, rel=1e-5, abs=1e-6)
    if po.ref_available():
        assert po.ref_dd_overlap(*[float(v) for v in args]) == pytest.approx(
            expected, rel=1e-5, abs=1e-6)


def _unit_image():
    # test_Siddon.cpp:48-75: 5x5x6 voxels, lengths 1.1 x 1.1 x 1.2, all ones.
    ip = po.ImageParams(5, 5, 6, 1.1, 1.1, 1.2)
    return ip, np.ones(ip.shape, np.float32)


def _fwd(ip, img, lors, **kw):
    return po.project(ip, po.Proj(threads=1, **kw), np.asarray(lors, np.float32),
                      image=img)


def test_siddon_isocenter_chords():
    ip, img = _unit_image()
    fr = ip.desc()
    fov = np.float32(max(np.float32(1.1) / 2, np.float32(1.1) / 2)) - \
        np.float32(np.float32(1.1) / 5) / np.float32(1000)
    lors = []
    for i in range(10):
        beta = 2 * math.pi * i / 9
        lors.append([-1.1 * math.cos(beta), -1.1 * math.sin(beta), 0,
                     1.1 * math.cos(beta), 1.1 * math.sin(beta), 0])
    v = _fwd(ip, img, lors)
    np.testing.assert_allclose(v, 2 * fov, rtol=1.2e-5)
    v64 = po.project(ip, po.Proj(threads=1), np.asarray(lors, np.float32),
                     image=img, precision="f64")
    np.testing.assert_allclose(v64, 2 * fov, rtol=1e-6)


def test_siddon_y_offset_chords_and_outside():
    ip, img = _unit_image()
    fov = float(np.float32(0.55) - np.float32(0.22) / np.float32(1000))
    lors, ref = [], []
    for i in range(10):
        y0 = 1.1 * i / 9 - 0.55
        lors.append([-1.1, y0, 0, 1.1, y0, 0])
        ref.append(2 * math.sqrt(max(0.0, fov * fov - y0 * y0)))
    np.testing.assert_allclose(_fwd(ip, img, lors), ref, rtol=1.2e-5, atol=1e-6)
    outside = [[1.1, 0, 0, 2.2, 0, 0], [2.2, 0, 0, 2.2, 1.1, 0],
               [-1.1, 0, 1.0001 * 0.6, 1.1, 0, 1.0001 * 0.6]]
    assert np.all(_fwd(ip, img, outside) == 0)


def test_siddon_axis_rays_and_z_rays():
    ip, img = _unit_image()
    fov = float(np.float32(0.55) - np.float32(0.22) / np.float32(1000))
    lors = [[0, 0, 1.2, 0, 0, -1.2], [0, -1.1, 0, 0, 1.1, 0],
            [-1.1, 0, 0, 1.1, 0, 0], [-1.1, -1.1, 0, 1.1, 1.1, 0]]
    ref = [1.2, 2 * fov, 2 * fov, 2 * fov]
    np.testing.assert_allclose(_fwd(ip, img, lors), ref, rtol=1.2e-5)
    rng = np.random.default_rng(5)
    z1 = rng.random(10) * 1.2 - 0.6
    z2 = rng.random(10) * 1.2 - 0.6
    lz = [[0, -fov, a, 0, fov, b] for a, b in zip(z1, z2)]
    np.testing.assert_allclose(_fwd(ip, img, lz),
                               np.sqrt(4 * fov * fov + (z2 - z1) ** 2), rtol=1e-4)


def test_siddon_regression_vertical_lor():
    # test_Siddon.cpp:504-530: 1x1x89 image, vertical LOR -> v * sz.
    ip = po.ImageParams(1, 1, 89, 1.0, 1.0, 89 * 2.0)
    img = np.full(ip.shape, 3.0, np.float32)
    v = _fwd(ip, img, [[0.0, 0.0, -200.0, 0.0, 0.0, 200.0]])
    np.testing.assert_allclose(v, 3.0 * 89 * 2.0, rtol=1e-5)


def test_siddon_adjoint_identity():
    rng = np.random.default_rng(3)
    lut = po.scanner_lut(SC)
    d1 = rng.integers(0, SC.num_dets, 3000)
    d2 = rng.integers(0, SC.num_dets, 3000)
    ok = d1 % 256 != d2 % 256
    lors, _ = po.lors_from_detpairs(lut, d1[ok], d2[ok])
    x = rng.random(IP.shape).astype(np.float32)
    y = rng.random(len(lors)).astype(np.float32)
    for tofw in (0.0, 214.0):
        tof = rng.normal(0, 200, len(lors)).astype(np.float32) if tofw else None
        pr = po.Proj(tof_fwhm_ps=tofw, tof_n_std=5)
        ax = po.project(IP, pr, lors, image=x, tof=tof, precision="f64")
        aty = po.project(IP, pr, lors, values=y.astype(np.float64), tof=tof,
                         forward=False, precision="f64")
        lhs = float(np.dot(ax, y))
        rhs = float(np.sum(aty * x))
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


# ----------------------------------------------------- golden (reference) --
def test_golden_lut_and_maps():
    assert np.array_equal(bits(po.scanner_lut(SC)), bits(GOLD["lut"]))
    bins = po.histo3d_bins(SC, GOLD["d1"], GOLD["d2"])
    assert np.array_equal(bins, GOLD["bins"])
    assert tuple(po.histo3d_dims(SC)) == tuple(int(v) for v in GOLD["histo_dims"])
    a, b = po.histo3d_detpairs(SC, GOLD["query_bins"])
    assert np.array_equal(a, GOLD["query_d1"]) and np.array_equal(b, GOLD["query_d2"])


def test_golden_siddon_forward_bitexact():
    lors, img, tof = GOLD["lors"], GOLD["image"], GOLD["tof"]
    v = po.project(IP, po.Proj(threads=1), lors, image=img)
    assert np.array_equal(bits(v), bits(GOLD["siddon_fwd"]))
    vt = po.project(IP, po.Proj(tof_fwhm_ps=214.0, tof_n_std=5, threads=1), lors,
                    image=img, tof=tof)
    assert np.array_equal(bits(vt), bits(GOLD["siddon_tof_fwd"]))


def test_golden_siddon_backward():
    lors, vals, tof = GOLD["lors"], GOLD["values"], GOLD["tof"]
    b = po.project(IP, po.Proj(threads=1), lors, values=vals, forward=False)
    np.testing.assert_allclose(b, GOLD["siddon_bwd"], rtol=1e-5, atol=1e-6)
    bt = po.project(IP, po.Proj(tof_fwhm_ps=214.0, tof_n_std=5, threads=1), lors,
                    values=vals, tof=tof, forward=False)
    np.testing.assert_allclose(bt, GOLD["siddon_tof_bwd"], rtol=1e-5, atol=1e-8)


def test_golden_dd_forward_bitexact():
    lors, ori, img, tof = GOLD["lors"], GOLD["orients"], GOLD["image"], GOLD["tof"]
    pr = po.Proj(projector="DD", crystal_z=4, crystal_trans=4, threads=1)
    assert np.array_equal(bits(po.project(IP, pr, lors, image=img, orients=ori)),
                          bits(GOLD["dd_fwd"]))
    pr = po.Proj(projector="DD", crystal_z=4, crystal_trans=4, tof_fwhm_ps=214.0,
                 tof_n_std=5, threads=1)
    assert np.array_equal(
        bits(po.project(IP, pr, lors, image=img, orients=ori, tof=tof)),
        bits(GOLD["dd_tof_fwd"]))


def test_mirror_vs_fp64_within_budget():
    lors, img, tof = GOLD["lors"], GOLD["image"], GOLD["tof"]
    pr = po.Proj(tof_fwhm_ps=214.0, tof_n_std=5)
    a = po.project(IP, pr, lors, image=img, tof=tof)
    b = po.project(IP, pr, lors, image=img, tof=tof, precision="f64")
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5


# ---------------------------------------------- live reference (optional) --
@needs_ref
def test_live_reference_siddon_random_bitexact():
    rng = np.random.default_rng(11)
    lut = po.scanner_lut(SC)
    d1 = rng.integers(0, SC.num_dets, 20000)
    d2 = rng.integers(0, SC.num_dets, 20000)
    ok = d1 % 256 != d2 % 256
    lors, _ = po.lors_from_detpairs(lut, d1[ok], d2[ok])
    ip = po.ImageParams(64, 64, 32, 128, 128, 64, 1.5, -2.0, 0.5)
    img = rng.random(ip.shape, dtype=np.float32)
    tof = rng.normal(0, 300, len(lors)).astype(np.float32)
    for tofw in (0.0, 214.0):
        t = tof if tofw else None
        a = po.project(ip, po.Proj(tof_fwhm_ps=tofw, tof_n_std=5), lors,
                       image=img, tof=t)
        b = po.ref_siddon(SC, ip, lors, image=img, tof=t, tof_fwhm_ps=tofw,
                          tof_n_std=5)
        assert np.array_equal(bits(a), bits(b))


@needs_ref
def test_live_reference_multiray_rand_r_stream():
    # CPU multi-ray: MultiRayGenerator draws rand_r(seed=13) offsets restarted
    # per LOR (ProjectorSiddon.cpp:258-264), so every LOR sees the same four
    # uniforms per extra ray.
    import ctypes
    libc = ctypes.CDLL(None)
    seed = ctypes.c_uint(13)
    nr = 4
    u = []
    for _ in range(4 * (nr - 1)):
        u.append(np.float32(np.float32(libc.rand_r(ctypes.byref(seed))) /
                            np.float32(2147483647)) - np.float32(0.5))
    rng = np.random.default_rng(12)
    lut = po.scanner_lut(SC)
    d1 = rng.integers(0, SC.num_dets, 3000)
    d2 = rng.integers(0, SC.num_dets, 3000)
    ok = d1 % 256 != d2 % 256
    lors, ori = po.lors_from_detpairs(lut, d1[ok], d2[ok])
    img = rng.random(IP.shape, dtype=np.float32)
    offs = np.tile(np.asarray(u, np.float32), (len(lors), 1))
    pr = po.Proj(num_rays=nr, crystal_z=4, crystal_trans=4)
    a = po.project(IP, pr, lors, image=img, orients=ori, ray_offsets=offs)
    b = po.ref_siddon(SC, IP, lors, image=img, orients=ori, num_rays=nr)
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)


@needs_ref
def test_live_reference_lm_to_histogram_bitexact():
    rng = np.random.default_rng(13)
    d1 = rng.integers(0, SC.num_dets, 200000).astype(np.uint32)
    d2 = rng.integers(0, SC.num_dets, 200000).astype(np.uint32)
    bins = po.histo3d_bins(SC, d1, d2)
    ok = (bins != np.iinfo(np.uint64).max) | (d1 == d2)
    h, bad = po.lm_to_histo3d(SC, d1[ok], d2[ok])
    assert bad == 0
    r, _ = po.ref_lm_to_histo3d(SC, d1[ok], d2[ok])
    assert np.array_equal(bits(h), bits(r))


# ------------------------------------------------------- image-space PSF --
@needs_ref
@pytest.mark.parametrize("adjoint", [False, True])
def test_psf_convolution_oracle_bitexact_vs_reference(adjoint):
    """The oracle's separable convolution (FP32, tap order, circular borders)
    against the reference's OperatorPsf::applyA / applyAH, bit for bit; the
    FP64 restatement within float rounding."""
    rng = np.random.default_rng(61)
    ip = po.ImageParams(20, 16, 12, 40, 32, 24, nt=2)
    img = rng.random((2, 12, 16, 20), dtype=np.float32)
    kx = rng.random(5).astype(np.float32)
    ky = rng.random(7).astype(np.float32)
    kz = rng.random(3).astype(np.float32)
    ref = po.ref_psf_convolve(ip, img, kx, ky, kz, adjoint=adjoint)
    f32 = po.psf_convolve(ip, img, kx, ky, kz, adjoint=adjoint)
    f64 = po.psf_convolve(ip, img, kx, ky, kz, adjoint=adjoint, precision="f64")
    assert np.array_equal(ref.view(np.uint32), f32.view(np.uint32))
    assert np.linalg.norm(f64 - ref) / np.linalg.norm(f64) < 1e-6


@needs_ref
def test_psf_gaussian_kernel_matches_reference():
    k = po.ref_psf_gaussian_kernel(1.7, 2.0, 7)
    x = (np.arange(7) - 3).astype(np.float32)
    mine = np.exp(-0.5 * (x * np.float32(2.0) / np.float32(1.7)) ** 2).astype(np.float32)
    mine /= mine.sum(dtype=np.float32)
    assert np.allclose(k, mine, rtol=1e-6)


# ------------------------------------------------------ low-rank images ----
def _lr_case(seed, n=6000, R=3, T=5):
    rng = np.random.default_rng(seed)
    lut = po.scanner_lut(SC)
    d1 = rng.integers(0, SC.num_dets, n)
    d2 = rng.integers(0, SC.num_dets, n)
    ok = d1 % 256 != d2 % 256
    lors, _ = po.lors_from_detpairs(lut, d1[ok], d2[ok])
    frames = rng.integers(0, T, len(lors)).astype(np.int32)
    W = rng.random((R,) + IP.shape[1:], dtype=np.float32)
    H = rng.random((R, T), dtype=np.float32)
    return lors, frames, W, H


@needs_ref
@pytest.mark.parametrize("tofw", [0.0, 214.0])
def test_lr_forward_is_forward_of_expanded_frames(tofw):
    """The reference's LR updater forward (rank sum at each crossing) equals,
    bit for bit, its plain forward projection of the expanded frames."""
    lors, frames, W, H = _lr_case(31)
    R, T = H.shape
    rng = np.random.default_rng(32)
    tof = rng.normal(0, 300, len(lors)).astype(np.float32) if tofw else None
    ipw = po.ImageParams(32, 32, 16, 128, 128, 64, nt=R)
    ipx = po.ImageParams(32, 32, 16, 128, 128, 64, nt=T)
    a = po.ref_siddon_lr(SC, ipw, lors, frames, H, image=W, tof=tof,
                         tof_fwhm_ps=tofw, tof_n_std=5)
    X = po.lr_expand(W, H)
    b = po.ref_siddon(SC, ipx, lors, image=X, tof=tof, tof_fwhm_ps=tofw,
                      tof_n_std=5, frames=frames)
    assert np.array_equal(bits(a), bits(b))


@needs_ref
def test_lr_backward_is_contraction_of_frame_backprojection():
    """The reference's LR updater back projection (rank atomics per crossing)
    equals the contraction of its frame-indexed back projection, up to the
    order of FP32 sums."""
    lors, frames, W, H = _lr_case(33)
    R, T = H.shape
    vals = np.random.default_rng(34).random(len(lors), dtype=np.float32)
    ipw = po.ImageParams(32, 32, 16, 128, 128, 64, nt=R)
    ipx = po.ImageParams(32, 32, 16, 128, 128, 64, nt=T)
    a = po.ref_siddon_lr(SC, ipw, lors, frames, H, values=vals, forward=False,
                         threads=1)
    E = po.ref_siddon(SC, ipx, lors, values=vals, frames=frames, forward=False,
                      threads=1)
    b = po.lr_contract_w_f64(E, H)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-6


def test_lr_oracle_expand_and_contractions_agree():
    """<A_lr W, y> identities of the restatement: the expansion and the two
    contractions are adjoint to each other in FP64."""
    rng = np.random.default_rng(35)
    R, T, J = 4, 7, 300
    W = rng.random((R, J), dtype=np.float32)
    H = rng.random((R, T), dtype=np.float32)
    E = rng.random((T, J), dtype=np.float32)
    X = po.lr_expand(W, H)
    lhs = float(np.sum(X.astype(np.float64) * E))
    rhs_w = float(np.sum(W.astype(np.float64) * po.lr_contract_w_f64(E, H)))
    rhs_h = float(np.sum(H.astype(np.float64) * po.lr_contract_h_f64(W, E)))
    assert abs(lhs - rhs_w) / lhs < 1e-6 and abs(lhs - rhs_h) / lhs < 1e-6
