"""Low-rank dynamic images on the device (yrtb_lr_*, LowRankProjector,
LREM_GPU) against the oracle's restatement and the reference's LR updater
and LREM_CPU (src/operators/ProjectorUpdater.cpp:228-280, src/recon/LREM*.cpp)."""
import numpy as np
import pytest
import torch

import pyoracle as po
import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import lrem

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


@pytest.mark.parametrize("R,T,J", [(1, 4, 1000), (3, 5, 4097), (8, 20, 20000),
                                   (17, 9, 3001), (32, 3, 777)])
def test_expand_bitexact_and_contractions(R, T, J):
    rng = np.random.default_rng(100 + R)
    W = rng.random((R, J), dtype=np.float32)
    H = rng.random((R, T), dtype=np.float32)
    E = rng.random((T, J), dtype=np.float32)
    dW, dH, dE = (torch.from_numpy(a).cuda() for a in (W, H, E))
    X = lrem.lr_expand(dW, dH).cpu().numpy()
    assert np.array_equal(bits(X), bits(po.lr_expand(W, H)))
    Wn = lrem.lr_contract_w(dE, dH).cpu().numpy()
    assert rel_l2(Wn, po.lr_contract_w_f64(E, H)) < 1e-6
    if R * T <= 2048:
        Hn = lrem.lr_contract_h(dW, dE, R).cpu().numpy()
        assert rel_l2(Hn, po.lr_contract_h_f64(W, E)) < 1e-7
        # fixed summation order: bit-identical on a second run
        Hn2 = lrem.lr_contract_h(dW, dE, R).cpu().numpy()
        assert np.array_equal(Hn, Hn2)


def test_update_h_matches_float_mirror():
    rng = np.random.default_rng(110)
    R, T = 6, 11
    H = rng.random((R, T), dtype=np.float32)
    Hn = rng.random((R, T)) * 3.0
    c = rng.random(R).astype(np.float32)
    c[2] = 0.0  # clamped to eps
    dH = torch.from_numpy(H.copy()).cuda()
    lrem.lr_update_h(dH, torch.from_numpy(Hn).cuda(), torch.from_numpy(c).cuda(),
                     1.19209e-07)
    eps = np.float32(1.19209e-07)
    inv = (np.float32(1) / np.maximum(c, eps)).astype(np.float32)
    expect = (H * (Hn.astype(np.float32) * inv[:, None]).astype(np.float32)).astype(np.float32)
    assert np.array_equal(bits(dH.cpu().numpy()), bits(expect))


def test_lr_argument_errors():
    W = torch.ones(33 * 10, device="cuda")
    H = torch.ones((33, 2), device="cuda")
    with pytest.raises(RuntimeError):
        lrem.lr_expand(W, H)
    W = torch.ones(30 * 10, device="cuda")
    E = torch.ones(100 * 10, device="cuda")
    with pytest.raises(RuntimeError):  # rank x frames > 2048
        lrem.lr_contract_h(W, E, 30)


def _dyn_events(n, seed, T, tof=False):
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c1()
    ev = S.generate_events(sc, n, seed, tof_fwhm_ps=214.0 if tof else None).numpy()
    rng = np.random.default_rng(seed + 1)
    ts = np.sort(rng.integers(0, 100000, len(ev["d1"]))).astype(np.uint32)
    fts = np.linspace(0, int(ts.max()) + 1, T + 1).astype(np.uint32)
    return sc, ev, ts, fts


@needs_ref
@pytest.mark.parametrize("tof", [False, True])
def test_lr_forward_backward_vs_reference_updater(tof):
    R, T = 4, 6
    sc, e, ts, fts = _dyn_events(30000, 120, T, tof)
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e.get("tof"), timestamps=ts)
    lm.addDynamicFraming(fts)
    rng = np.random.default_rng(121)
    W = rng.random(ip.shape, dtype=np.float32)
    H = rng.random((R, T), dtype=np.float32)
    op = yrt.ProjectionOper(sc, ip, lm, updater_type="LR", H_basis=H,
                            tof_width_ps=214.0 if tof else None,
                            tof_n_std=5 if tof else 0)
    y = op.A(W)
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    lors, _ = po.lors_from_detpairs(po.scanner_lut(osc), e["d1"], e["d2"])
    frames = lm.dynamicFrames
    y_ref = po.ref_siddon_lr(osc, oip, lors, frames, H, image=W, tof=e.get("tof"),
                             tof_fwhm_ps=214.0 if tof else 0.0, tof_n_std=5)
    assert np.max(np.abs(y - y_ref)) <= 1e-5 * max(1.0, float(np.max(np.abs(y_ref))))
    vals = rng.random(len(y), dtype=np.float32)
    bw = op.At(vals)
    bw_ref = po.ref_siddon_lr(osc, oip, lors, frames, H, values=vals, forward=False,
                              tof=e.get("tof"), tof_fwhm_ps=214.0 if tof else 0.0,
                              tof_n_std=5)
    assert rel_l2(bw, bw_ref) < 1e-5
    # adjoint pair
    lhs = float(np.dot(y.astype(np.float64), vals))
    rhs = float(np.sum(W.astype(np.float64) * bw))
    assert abs(lhs - rhs) / abs(rhs) < 1e-5


@needs_ref
def test_lr_backward_h_is_gradient_of_forward_in_h():
    """<A_lr(W; H) , y> is linear in H: its H-gradient is the H back projection."""
    R, T = 3, 5
    sc, e, ts, fts = _dyn_events(20000, 122, T)
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], timestamps=ts)
    lm.addDynamicFraming(fts)
    rng = np.random.default_rng(123)
    W = rng.random(ip.shape, dtype=np.float32)
    H = rng.random((R, T), dtype=np.float32)
    vals = rng.random(len(e["d1"]), dtype=np.float32)
    op_h = yrt.ProjectionOper(sc, ip, lm, updater_type="LR", H_basis=H, update_H=True)
    G = op_h.At(vals, W=W)
    lhs = float(np.dot(yrt.ProjectionOper(sc, ip, lm, updater_type="LR",
                                          H_basis=H).A(W).astype(np.float64), vals))
    assert abs(float(np.sum(G * H)) - lhs) / abs(lhs) < 1e-5


@needs_ref
@pytest.mark.parametrize("tof", [False, True])
def test_lrem_update_w_vs_reference(tof):
    R, T = 3, 5
    sc, e, ts, fts = _dyn_events(60000, 130, T, tof)
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    rng = np.random.default_rng(131)
    H = (0.2 + rng.random((R, T))).astype(np.float32)
    osem = yrt.createOSEM(sc, True, isLowRank=True)
    osem.setImageParams(ip)
    osem.setProjectorUpdaterType("LR")
    osem.setHBasisFromNumpy(H)
    assert np.array_equal(osem.getHBasisNumpy(), H)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 2
    osem.setListModeEnabled(True)
    if tof:
        osem.addTOF(214.0, 5)
    sens = osem.generateSensitivityImages()
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], tof=e.get("tof"), timestamps=ts)
    lm.addDynamicFraming(fts)
    osem.setDataInput(lm)
    W = osem.reconstruct().cpu().numpy()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    s0 = sens[0].cpu().numpy()
    W_ref, H_after, _ = po.ref_lrem_listmode(
        osc, oip, s0, e["d1"], e["d2"], ts, fts, H, tof=e.get("tof"),
        iterations=2, subsets=2, tof_fwhm_ps=214.0 if tof else 0.0,
        tof_n_std=5 if tof else 0)
    assert np.array_equal(H_after, H)
    assert rel_l2(W, W_ref) < 1e-4


@needs_ref
def test_lrem_update_h_vs_reference():
    R, T = 3, 6
    sc, e, ts, fts = _dyn_events(60000, 140, T)
    ip = yrt.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    rng = np.random.default_rng(141)
    H0 = (0.2 + rng.random((R, T))).astype(np.float32)
    W0 = (0.5 + rng.random(ip.shape)).astype(np.float32)
    H = H0.copy()
    osem = yrt.createOSEM(sc, True, isLowRank=True)
    osem.setImageParams(ip)
    osem.setProjectorUpdaterType("LR")
    osem.setHBasisFromNumpy(H)
    osem.setUpdateH(True)
    osem.setInitialEstimate(W0)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 3
    osem.setListModeEnabled(True)
    sens = osem.generateSensitivityImages()
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"], timestamps=ts)
    lm.addDynamicFraming(fts)
    osem.setDataInput(lm)
    W = osem.reconstruct().cpu().numpy()
    osc = po.Scanner(*SC_ARGS)
    oip = po.ImageParams(32, 32, 16, 256, 256, 128, nt=R)
    W_ref, H_ref, _ = po.ref_lrem_listmode(
        osc, oip, sens[0].cpu().numpy(), e["d1"], e["d2"], ts, fts, H0,
        update_h=True, init=W0, iterations=2, subsets=3)
    s0 = sens[0].cpu().numpy().reshape(-1)
    # W stays the (masked) initial estimate; H is updated in the bound array
    expect_W = np.where(np.broadcast_to(s0 > 0, (R, s0.size)), W0.reshape(R, -1), 0)
    assert np.array_equal(bits(W.reshape(R, -1)), bits(expect_W))
    assert np.array_equal(bits(W_ref.reshape(R, -1)), bits(expect_W))
    assert not np.allclose(H, H0)
    assert rel_l2(H, H_ref) < 1e-4
