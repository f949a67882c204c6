"""Edge cases of the projection path through the C ABI, against the oracle.

Empty event sets, ragged event counts around the warp and block sizes,
degenerate and missing rays, TOF windows outside the image, strided ranges
and an all-zero histogram.  Tolerances: bit-exact for non-TOF mirror-mode
forward projections and for zeros; back projections 1e-6 relative L2 against
the FP32 (mirror) oracle and 1e-4 against FP64.
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


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def projector(tof=None):
    sc = yrt.Scanner("t", *SC_ARGS)
    ip = yrt.ImageParams(*IP_ARGS)
    pp = yrt.ProjectorParams(sc)
    if tof:
        pp.addTOF(*tof)
    return sc, ip, yrt.DeviceProjector(sc, ip, pp)


def image(ip, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.5, 1.5, ip.shape).astype(np.float32)


def oracle_forward(lors, img, tof=None, tof_args=None, precision="f32"):
    pr = po.Proj(tof_fwhm_ps=tof_args[0] if tof_args else 0.0,
                 tof_n_std=tof_args[1] if tof_args else 0)
    return po.project(po.ImageParams(*IP_ARGS), pr, lors, image=img, tof=tof,
                      precision=precision)


def test_empty_event_set_is_a_no_op():
    sc, ip, p = projector((214.0, 5))
    e32 = np.zeros(0, np.uint32)
    ev = yrt.DeviceEvents.from_arrays(e32, e32, tof=np.zeros(0, np.float32))
    img = torch.from_numpy(image(ip, 1)).cuda()
    assert p.forward(img, ev).numel() == 0
    b = p.backward(torch.zeros(0, device="cuda"), ev)
    assert torch.count_nonzero(b) == 0
    em = torch.zeros(ip.shape, device="cuda")
    p.em_step(img, em, ev)
    assert torch.count_nonzero(em) == 0
    mu = torch.full((ip.numVoxels,), 0.0096, device="cuda")
    assert p.attenuation_factors(mu, ip, ev).numel() == 0
    ordered, offs = p.order_events(ev, 4)
    assert ordered.count == 0 and np.all(offs == 0)
    assert p.take_event_errors() == 0


@pytest.mark.parametrize("n", [1, 31, 32, 33, 255, 257, 1001])
def test_ragged_event_counts_vs_oracle(n):
    sc, ip, p = projector()
    rng = np.random.default_rng(100 + n)
    osc = po.Scanner(*SC_ARGS)
    d1 = rng.integers(0, osc.num_dets, 4 * n + 8).astype(np.uint32)
    d2 = rng.integers(0, osc.num_dets, 4 * n + 8).astype(np.uint32)
    keep = (d1 % 256) != (d2 % 256)
    d1, d2 = d1[keep][:n], d2[keep][:n]
    img = image(ip, n)
    ev = yrt.DeviceEvents.from_arrays(d1, d2)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    lors, _ = po.lors_from_detpairs(po.scanner_lut(osc), d1, d2)
    assert np.array_equal(bits(v), bits(oracle_forward(lors, img)))
    y = rng.uniform(0.1, 1.0, n).astype(np.float32)
    b = p.backward(torch.from_numpy(y).cuda(), ev).cpu().numpy()
    oip = po.ImageParams(*IP_ARGS)
    # Mirror mode reproduces the reference's FP32 weights: against the FP32
    # oracle only the atomics' order differs; against FP64 the image budget.
    b32 = po.project(oip, po.Proj(), lors, values=y, forward=False)
    b64 = po.project(oip, po.Proj(), lors, values=y.astype(np.float64),
                     forward=False, precision="f64")
    assert rel_l2(b, b32) < 1e-6
    assert rel_l2(b, b64) < 1e-4


def test_degenerate_and_missing_rays_vs_oracle():
    # Zero-length LORs (both endpoints equal), LORs that miss the image
    # (a chord outside the 64 mm half-width), a ray along an image axis
    # through voxel corners, and a ray parallel to z: the forward
    # projections equal the mirror oracle's bit for bit (zeros included).
    sc, ip, p = projector()
    img = image(ip, 7)
    lors = np.array([
        [10.0, 5.0, 3.0, 10.0, 5.0, 3.0],          # zero length
        [-300.0, 90.0, 0.0, 300.0, 90.0, 0.0],     # misses (y beyond 64 mm)
        [-300.0, 0.0, 0.0, 300.0, 0.0, 0.0],       # along x through corners
        [0.0, -300.0, 8.0, 0.0, 300.0, 8.0],       # along y through corners
        [3.0, 5.0, -300.0, 3.0, 5.0, 300.0],       # parallel to z
        [-300.0, -300.0, -40.0, 300.0, 300.0, 40.0],
    ], np.float32)
    ev = yrt.DeviceEvents.from_arrays(lor=lors)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    ref = oracle_forward(lors, img)
    assert np.array_equal(bits(v), bits(ref))
    assert v[0] == 0.0 and v[1] == 0.0 and v[2] > 0.0 and v[4] > 0.0


def test_tof_windows_outside_the_image():
    # TOF offsets of +-50 ns put the kernel's window at the LOR's ends, far
    # outside the 128 mm image: nothing is projected, as in the oracle.
    sc, ip, p = projector((214.0, 5))
    osc = po.Scanner(*SC_ARGS)
    d1 = np.array([0, 64, 128, 200], np.uint32)
    d2 = np.array([128, 192, 0, 72], np.uint32)
    tof = np.array([5e4, -5e4, 5e4, 0.0], np.float32)
    img = image(ip, 8)
    ev = yrt.DeviceEvents.from_arrays(d1, d2, tof=tof)
    v = p.forward(torch.from_numpy(img).cuda(), ev).cpu().numpy()
    lors, _ = po.lors_from_detpairs(po.scanner_lut(osc), d1, d2)
    ref = oracle_forward(lors, img, tof=tof, tof_args=(214.0, 5), precision="f64")
    assert np.all(v[:3] == 0.0) and np.all(ref[:3] == 0.0)
    assert v[3] > 0.0 and abs(v[3] - ref[3]) <= 1e-5 * ref[3]


def test_strided_range_projects_only_its_events():
    sc, ip, p = projector()
    rng = np.random.default_rng(9)
    osc = po.Scanner(*SC_ARGS)
    n = 5000
    d1 = rng.integers(0, osc.num_dets, 2 * n).astype(np.uint32)
    d2 = rng.integers(0, osc.num_dets, 2 * n).astype(np.uint32)
    keep = (d1 % 256) != (d2 % 256)
    d1, d2 = d1[keep][:n], d2[keep][:n]
    img = image(ip, 10)
    ev = yrt.DeviceEvents.from_arrays(d1, d2)
    start, stride, count = 3, 7, 500
    out = torch.full((n,), -1.0, device="cuda")
    p.forward(torch.from_numpy(img).cuda(), ev, out=out,
              rng=L.yrtb_range(start, stride, count))
    v = out.cpu().numpy()
    idx = start + stride * np.arange(count)
    lors, _ = po.lors_from_detpairs(po.scanner_lut(osc), d1[idx], d2[idx])
    assert np.array_equal(bits(v[idx]), bits(oracle_forward(lors, img)))
    mask = np.ones(n, bool)
    mask[idx] = False
    assert np.all(v[mask] == -1.0)


def test_all_zero_histogram_selects_no_bins():
    sc, ip, p = projector()
    h = yrt.Histogram3D(sc)
    meas = torch.zeros(h.histoSize, device="cuda")
    img = torch.from_numpy(image(ip, 11)).cuda()
    nps = h.numPhi // 4 + (1 if 1 + (h.numPhi // 4) * 4 < h.numPhi else 0)
    bins = p.histo3d_subset_nonzero(meas, 4, 1, h.numR * nps * h.numZBin)
    assert bins.numel() == 0
    em = torch.zeros(ip.shape, device="cuda")
    p.em_step_histo3d(img, em, meas, 4, 1, bins=bins)
    p.em_step_histo3d(img, em, meas, 4, 1)
    assert torch.count_nonzero(em) == 0


@pytest.mark.parametrize("precision", [L.YRTB_MIRROR, L.YRTB_COMPENSATED])
def test_attenuation_strided_range_matches_full_range(precision):
    # The attenuation walks run grouped by their length through a
    # permutation of the range's items: a strided range gives, event by
    # event, the factors of the full range (bit for bit) and writes nothing
    # else.
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ip = yrt.ImageParams(64, 64, 32, 256, 256, 128)
    pp = yrt.ProjectorParams(sc)
    pp.precision = precision
    p = yrt.DeviceProjector(sc, ip, pp)
    e = S.generate_events(sc, 20000, 93).numpy()
    ev = yrt.DeviceEvents.from_arrays(e["d1"], e["d2"])
    mu = S.Phantom(cyl_half_length=32).mu_image(ip, device="cuda").reshape(-1).contiguous()
    full = p.attenuation_factors(mu, ip, ev).cpu().numpy()
    out = torch.full((ev.count,), -1.0, device="cuda")
    start, stride, count = 5, 3, 4000
    p.attenuation_factors(mu, ip, ev, out=out, rng=L.yrtb_range(start, stride, count))
    v = out.cpu().numpy()
    idx = start + stride * np.arange(count)
    assert np.array_equal(bits(v[idx]), bits(full[idx]))
    mask = np.ones(ev.count, bool)
    mask[idx] = False
    assert np.all(v[mask] == -1.0)
    assert np.any(full < 1.0)
