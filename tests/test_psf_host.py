"""Host side of the image-space PSF: Gaussian kernels against the reference
OperatorPsf::createGaussianKernel1D (src/operators/OperatorPsf.cpp:158-190)
and the CSV layout read by OperatorPsf(fname) (:219-270)."""
import numpy as np
import pytest

import pyoracle as po
from pyyrtpet_b200.psf import OperatorPsfDevice, write_image_psf_csv

needs_ref = pytest.mark.skipif(not po.ref_available(),
                               reason="reference library not built")


@needs_ref
@pytest.mark.parametrize("sigma,vox,size", [(1.7, 2.0, 7), (0.9, 2.0, 3),
                                            (3.3, 2.5, 9), (2.0, 2.0, 0),
                                            (1.2, 0.5, 0)])
def test_gaussian_kernel_matches_reference(sigma, vox, size):
    mine = OperatorPsfDevice.createGaussianKernel1D(sigma, vox, size or None)
    ref = po.ref_psf_gaussian_kernel(sigma, vox, size)
    if len(ref) % 2 == 1:
        assert len(mine) == len(ref)
        # exp may differ in the last place between libms (and so the sum)
        assert np.allclose(mine, ref, rtol=1e-6, atol=0)
    else:
        # Even default sizes become odd: the reference's convolution reads
        # 2 (size/2) + 1 taps, one past the end of an even kernel.
        assert len(mine) == len(ref) + 1


def test_gaussian_kernel_default_size_and_normalisation():
    k = OperatorPsfDevice.createGaussianKernel1D(2.0, 1.0)
    assert len(k) == 11  # rint(5 * 2 / 1) = 10, made odd
    assert abs(float(k.sum(dtype=np.float64)) - 1.0) < 1e-6
    assert np.array_equal(k, k[::-1])
    with pytest.raises(RuntimeError):
        OperatorPsfDevice.createGaussianKernel1D(-1.0, 1.0)


def test_image_psf_csv_layout(tmp_path):
    fname = str(tmp_path / "p.csv")
    kx = np.array([0.25, 0.5, 0.25], np.float32)
    ky = np.array([0.1, 0.2, 0.4, 0.2, 0.1], np.float32)
    kz = np.array([1.0], np.float32)
    write_image_psf_csv(fname, kx, ky, kz)
    rows = [r.split(",") for r in open(fname).read().strip().split("\n")]
    assert len(rows) == 4
    assert [int(v) for v in rows[3]] == [3, 5, 1]
    assert np.array_equal(np.array(rows[1], np.float32), ky)


# ------------------------------------------- spatially variant image PSF --
def _varpsf_csv(path, rows, rng_gap_nstd):
    with open(path, "w") as f:
        for r in rng_gap_nstd + rows:
            f.write(",".join(f"{float(v):.9g}" for v in r) + "\n")


@needs_ref
@pytest.mark.parametrize("values", [[1.3, 0.8, 2.1], [0.7, 0.9, 1.2, 1.9, 2.2, 2.4, 0.35]])
def test_varpsf_gaussian_kernels_bitexact_vs_reference(values):
    from pyyrtpet_b200.core import ImageParams
    from pyyrtpet_b200.psf import _gaussian_kernel
    ip = ImageParams(40, 36, 20, 80.0, 75.6, 50.0)
    oip = po.ImageParams(40, 36, 20, 80.0, 75.6, 50.0)
    nstd = [4.0, 3.5, 4.0]
    mine = _gaussian_kernel(values, nstd, ip)
    ref, half = po.ref_varpsf_gaussian_kernel(values, nstd, oip)
    assert mine.half_sizes == half
    assert np.array_equal(mine.weights.view(np.uint32), ref.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("gap", [4.0, 4.5])
@pytest.mark.parametrize("adjoint", [False, True])
def test_varpsf_fp64_restatement_vs_reference(tmp_path, gap, adjoint):
    """The FP64 restatement of varconvolve (kernel choice by nearest LUT
    entry, circular borders) against the reference operator."""
    from pyyrtpet_b200.core import ImageParams
    from pyyrtpet_b200.psf import _gaussian_kernel
    nx, ny, nz = 14, 12, 9
    ip = ImageParams(nx, ny, nz, 14.0, 13.2, 11.7)
    oip = po.ImageParams(nx, ny, nz, 14.0, 13.2, 11.7)
    rng = np.random.default_rng(91)
    rg = [[7.0, 7.0, 6.0], [gap, gap, gap], [3.0, 3.0, 3.0]]
    dims = [int(np.floor(np.float32(r) / np.float32(gap))) + 1 for r in rg[0]]
    rows = [list(rng.uniform(0.4, 1.2, 3)) for _ in range(dims[0] * dims[1] * dims[2])]
    csv = str(tmp_path / "var.csv")
    _varpsf_csv(csv, rows, rg)
    ks = [_gaussian_kernel(r, rg[2], ip) for r in rows]
    img = rng.random((nz, ny, nx), dtype=np.float32)
    ref = po.ref_varpsf_apply(oip, csv, img, adjoint=adjoint, threads=1)
    mine = po.varpsf_apply_f64(oip, img, [k.weights for k in ks],
                               [k.half_sizes for k in ks], rg[0] + rg[1], adjoint=adjoint)
    assert np.linalg.norm(mine - ref) / np.linalg.norm(ref) < 1e-6
