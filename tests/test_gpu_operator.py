"""The projection operator (ProjectionOper A / At) on list-mode and histogram
data, as the reference's integration helpers check it
(integration_tests/helper.py:43-89): the subsets' projections add up to the
full projection, and each operator satisfies <A x, y> = <x, A^T y>.

Tolerances: the subset sum is bit-exact here (every bin's projection is
computed the same way whatever subset it is in; the reference allows
allclose); the adjoint identity to 1e-6 relative in FP64 (the reference
allows 1e-3).  Multi-ray offsets follow an event's index in the call, as in
the reference device path, so for multi-ray only the adjoint identity holds
per subset.
"""
import numpy as np
import pytest
import torch  # noqa: F401  (CUDA context for the operator)

import pyyrtpet_b200 as yrt

pytestmark = pytest.mark.gpu

SC_ARGS = ("s", 20, 4, 4, 10, 150, 64, 5, 1, 4, 2, 1)   # 64 x 5 crystals, every ring difference
IP_ARGS = (32, 32, 8, 160, 160, 20)


def _data(kind, tof):
    sc = yrt.Scanner(*SC_ARGS)
    rng = np.random.default_rng(61)
    if kind == "histogram":
        return sc, yrt.Histogram3D(sc)
    n = 20000
    d1 = rng.integers(0, sc.getNumDets(), 3 * n).astype(np.uint32)
    d2 = rng.integers(0, sc.getNumDets(), 3 * n).astype(np.uint32)
    keep = (d1 % 64) != (d2 % 64)
    lm = yrt.ListModeLUT(sc, tof, False)
    lm.allocate(n)
    lm.d1[:] = d1[keep][:n]
    lm.d2[:] = d2[keep][:n]
    if tof:
        lm.tof[:] = rng.normal(0, 150, n).astype(np.float32)
    return sc, lm


CASES = [("listmode", "Siddon", False, 1), ("listmode", "Siddon", True, 1),
         ("listmode", "DD", False, 1), ("listmode", "Siddon", False, 4),
         ("histogram", "Siddon", False, 1), ("histogram", "DD", False, 1),
         ("histogram", "Siddon", False, 4)]


@pytest.mark.parametrize("kind,projector,tof,rays", CASES)
def test_projection_oper_subsets_and_adjoint(kind, projector, tof, rays):
    sc, data = _data(kind, tof)
    ip = yrt.ImageParams(*IP_ARGS)
    kw = dict(projector=projector, num_rays=rays)
    if tof:
        kw.update(tof_width_ps=214.0, tof_n_std=5)
    rng = np.random.default_rng(62)
    x = rng.random((ip.nz, ip.ny, ip.nx)).astype(np.float32)
    y = rng.random(data.count()).astype(np.float32)
    k = yrt.ProjectionOper(sc, ip, data, **kw)
    Ax = k.A(x)
    assert Ax.shape == (data.count(),) and np.count_nonzero(Ax) > 0
    Aty = k.At(y)
    lhs = float(np.dot(Ax.astype(np.float64), y))
    rhs = float(np.sum(x.astype(np.float64) * Aty.reshape(x.shape)))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    S = 4
    Ax_sub = np.zeros_like(Ax)
    for s in range(S):
        ks = yrt.ProjectionOper(sc, ip, data, idx_subset=s, num_subsets=S, **kw)
        Ax_s = ks.A(x)
        Ax_sub += Ax_s
        Aty_s = ks.At(y)
        lhs = float(np.dot(Ax_s.astype(np.float64), y))
        rhs = float(np.sum(x.astype(np.float64) * Aty_s.reshape(x.shape)))
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    if rays == 1:
        assert np.array_equal(Ax_sub, Ax)


@pytest.mark.parametrize("kind", ["listmode", "histogram"])
def test_operator_projector_device_reference_signatures(kind):
    # OperatorProjectorDevice with the reference's pybind signatures
    # (src/operators/OperatorProjectorDevice.cu:26-90): applyA(img, proj)
    # writes into a ProjectionList (entries of other subsets untouched),
    # applyAH(proj, img) adds into img; same values as ProjectionOper.
    sc, data = _data(kind, False)
    ip = yrt.ImageParams(*IP_ARGS)
    pp = yrt.ProjectorParams(sc)
    it = data.getBinIter(3, 1)
    op = yrt.OperatorProjectorDevice.create(pp, it, img_params=ip)
    rng = np.random.default_rng(62)
    x = torch.from_numpy(rng.random(ip.shape, dtype=np.float32)).cuda()
    pl = yrt.ProjectionListOwned(data)
    pl.allocate()
    pl.clearProjections(-1.0)
    op.applyA(x, pl)
    A = yrt.ProjectionOper(sc, ip, data, idx_subset=1, num_subsets=3)
    ref = A.A(x.cpu().numpy())
    idx = np.asarray(it.indices()) if kind == "histogram" else np.arange(1, data.count(), 3)
    got = pl.getProjectionsArray()
    assert np.array_equal(got[idx], ref[idx])
    outside = np.setdiff1d(np.arange(data.count()), idx)
    assert np.all(got[outside] == -1.0)
    y = yrt.ProjectionListOwned(data)
    y.allocate()
    y.values.copy_(torch.from_numpy(rng.random(data.count(), dtype=np.float32)))
    img = torch.zeros(ip.shape, device="cuda")
    op.applyAH(y, img)
    bp = A.At(y.getProjectionsArray())
    assert np.allclose(img.cpu().numpy(), bp, rtol=1e-5, atol=1e-6)
    with pytest.raises(RuntimeError):
        op.applyA(x, data)          # a ProjectionList receives the values
