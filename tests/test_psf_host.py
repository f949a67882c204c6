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
