"""Image-space PSF mirroring the reference OperatorPsf / OperatorPsfDevice
(include/yrt-pet/operators/OperatorPsf.hpp:19-70,
src/operators/OperatorPsf.cpp:128-375): a spatially invariant, separable
kernel (one odd-length 1-D kernel per axis) applied by libyrtb
(yrtb_psf_apply) with circular borders; applyAH uses the flipped kernels.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from .core import ImageParams, _stream

SIGMA_TO_FWHM = 2.354820045031  # 2 sqrt(2 ln 2)


class OperatorPsfDevice:
    def __init__(self, *args):
        """OperatorPsfDevice(), OperatorPsfDevice(fname) or
        OperatorPsfDevice(kernel_x, kernel_y, kernel_z)."""
        self._h = None
        self._k = [np.zeros(1, np.float32)] * 3
        if len(args) == 1:
            self.readFromFile(args[0])
        elif len(args) == 3:
            self._set(*args)
        elif args:
            raise RuntimeError("OperatorPsfDevice(fname) or (kernel_x, kernel_y, kernel_z)")

    # -------------------------------------------------------- kernels ------
    def _set(self, kx, ky, kz):
        ks = [np.ascontiguousarray(k, np.float32).ravel() for k in (kx, ky, kz)]
        for k in ks:
            if k.size % 2 == 0:
                raise RuntimeError("Kernel size must be odd")
        h = ctypes.c_void_p()
        L.check(L.lib().yrtb_psf_create(ks[0].ctypes.data, ks[0].size,
                                        ks[1].ctypes.data, ks[1].size,
                                        ks[2].ctypes.data, ks[2].size,
                                        ctypes.byref(h)))
        self._release()
        self._h = h
        self._k = ks

    def _release(self):
        if self._h is not None:
            L.lib().yrtb_psf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    @staticmethod
    def createGaussianKernel1D(sigma: float, voxelSize: float,
                               kernelSize: Optional[int] = None) -> np.ndarray:
        """exp(-(x v / sigma)^2 / 2) at x = i - size/2, normalised to sum 1
        (OperatorPsf::createGaussianKernel1D, OperatorPsf.cpp:128-157).  The
        default size is rint(5 sigma / v), made odd when even: the reference
        convolves 2 (size/2) + 1 taps, one past an even-sized kernel."""
        if sigma < 0:
            raise RuntimeError("Gaussian Sigma or FWHM cannot be null or negative")
        if voxelSize < 0:
            raise RuntimeError("Voxel size cannot be null or negative")
        f32 = np.float32
        size = int(kernelSize) if kernelSize else int(
            np.rint(f32(5) * f32(sigma) / f32(voxelSize)))
        if size % 2 == 0:
            size += 1
        x = (np.arange(size) - size // 2).astype(f32)
        k = np.exp(f32(-0.5) * np.square(x * f32(voxelSize) / f32(sigma)), dtype=f32)
        total = f32(0)
        for v in k:  # sequential FP32 sum, as std::accumulate
            total = f32(total + v)
        return (k / total).astype(f32)

    @classmethod
    def createGaussianFromSigma(cls, sigmaX, sigmaY, sigmaZ, vx, vy, vz,
                                kernelSizeX=None, kernelSizeY=None, kernelSizeZ=None):
        return cls(cls.createGaussianKernel1D(sigmaX, vx, kernelSizeX),
                   cls.createGaussianKernel1D(sigmaY, vy, kernelSizeY),
                   cls.createGaussianKernel1D(sigmaZ, vz, kernelSizeZ))

    @classmethod
    def createGaussianFromFWHM(cls, fwhmX, fwhmY, fwhmZ, vx, vy, vz,
                               kernelSizeX=None, kernelSizeY=None, kernelSizeZ=None):
        f = np.float32(SIGMA_TO_FWHM)
        return cls.createGaussianFromSigma(
            np.float32(fwhmX) / f, np.float32(fwhmY) / f, np.float32(fwhmZ) / f,
            vx, vy, vz, kernelSizeX, kernelSizeY, kernelSizeZ)

    def readFromFile(self, fname: str):
        """CSV: kernel x, kernel y, kernel z, then the three sizes
        (OperatorPsf::readFromFileInternal, OperatorPsf.cpp:176-224)."""
        rows = []
        with open(fname) as f:
            for line in f:
                vals = [v for v in line.replace(",", " ").split() if v]
                if vals:
                    rows.append([float(v) for v in vals])
        if len(rows) < 4:
            raise RuntimeError(f"Error reading image-space PSF file '{fname}'")
        sizes = [int(v) for v in rows[3][:3]]
        for s in sizes:
            if s % 2 == 0:
                raise RuntimeError("Kernel size must be odd")
        self._set(*(np.asarray(rows[a][:sizes[a]], np.float32) for a in range(3)))

    def getKernelX(self):
        return self._k[0].copy()

    def getKernelY(self):
        return self._k[1].copy()

    def getKernelZ(self):
        return self._k[2].copy()

    def getKernelXFlipped(self):
        return self._k[0][::-1].copy()

    def getKernelYFlipped(self):
        return self._k[1][::-1].copy()

    def getKernelZFlipped(self):
        return self._k[2][::-1].copy()

    # -------------------------------------------------------- operator -----
    @staticmethod
    def _params(img: torch.Tensor, params: Optional[ImageParams]):
        if params is not None:
            return params
        sh = img.shape
        if img.dim() == 3:
            nz, ny, nx = sh
            nt = 1
        elif img.dim() == 4:
            nt, nz, ny, nx = sh
        else:
            raise RuntimeError("images must be (nz, ny, nx) or (nt, nz, ny, nx)")
        return ImageParams(nx, ny, nz, float(nx), float(ny), float(nz), nt=nt)

    def _apply(self, img_in, img_out, adjoint, params=None, tmp=None):
        if self._h is None:
            raise RuntimeError("PSF kernels not set")
        for t in (img_in, img_out):
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                raise RuntimeError("images must be contiguous float32 CUDA tensors")
        if img_in.numel() != img_out.numel():
            raise RuntimeError("Dimensions mismatch between the two images")
        ip = self._params(img_in, params)
        L.check(L.lib().yrtb_psf_apply(self._h, img_in.data_ptr(), img_out.data_ptr(),
                                       ctypes.byref(ip._c()), int(adjoint),
                                       None if tmp is None else tmp.data_ptr(),
                                       _stream()))
        return img_out

    def applyA(self, img_in, img_out, params: Optional[ImageParams] = None):
        return self._apply(img_in, img_out, False, params)

    def applyAH(self, img_in, img_out, params: Optional[ImageParams] = None):
        return self._apply(img_in, img_out, True, params)

    def convolve(self, img_in, img_out, kernelX: Sequence[float],
                 kernelY: Sequence[float], kernelZ: Sequence[float],
                 params: Optional[ImageParams] = None):
        return OperatorPsfDevice(kernelX, kernelY, kernelZ).applyA(img_in, img_out, params)

    @property
    def handle(self):
        return self._h


def write_image_psf_csv(fname: str, kernel_x, kernel_y, kernel_z):
    """Writes the image-space PSF CSV read by OperatorPsf(fname): one row per
    axis kernel (x, y, z), then a row with the three sizes."""
    ks = [np.ascontiguousarray(k, np.float32).ravel() for k in (kernel_x, kernel_y, kernel_z)]
    with open(fname, "w") as f:
        for k in ks:
            f.write(",".join(f"{float(v):.9g}" for v in k) + "\n")
        f.write(",".join(str(k.size) for k in ks) + "\n")


# ------------------------------------------- spatially variant image PSF ---
class ConvolutionKernel:
    """One kernel of a variant PSF LUT: weights (2hz+1, 2hy+1, 2hx+1)."""

    def __init__(self, weights, half_sizes=None):
        w = np.ascontiguousarray(weights, np.float32)
        if w.ndim != 3 or any(n % 2 == 0 for n in w.shape):
            raise RuntimeError("kernel must be 3-D with odd sizes")
        self.weights = w
        self.half_sizes = (w.shape[2] // 2, w.shape[1] // 2, w.shape[0] // 2)

    def getHalfSizeX(self):
        return self.half_sizes[0]

    def getHalfSizeY(self):
        return self.half_sizes[1]

    def getHalfSizeZ(self):
        return self.half_sizes[2]

    def getArray(self):
        return self.weights.copy()


def _gaussian_kernel(values, nstd, params: ImageParams) -> ConvolutionKernel:
    sig = np.ascontiguousarray(values, np.float32)
    ns = np.ascontiguousarray(nstd, np.float32)
    half = np.zeros(3, np.int32)
    size = ctypes.c_uint64()
    ip = params._c()
    L.check(L.lib().yrtb_varpsf_gaussian_kernel(sig.ctypes.data, len(sig), ns.ctypes.data,
                                                ctypes.byref(ip), None, 0, half.ctypes.data,
                                                ctypes.byref(size)))
    out = np.zeros(size.value, np.float32)
    L.check(L.lib().yrtb_varpsf_gaussian_kernel(sig.ctypes.data, len(sig), ns.ctypes.data,
                                                ctypes.byref(ip), out.ctypes.data, out.size,
                                                half.ctypes.data, ctypes.byref(size)))
    hx, hy, hz = (int(v) for v in half)
    return ConvolutionKernel(out.reshape(2 * hz + 1, 2 * hy + 1, 2 * hx + 1))


class ConvolutionKernelGaussian(ConvolutionKernel):
    """ConvolutionKernelGaussian (src/operators/OperatorVarPsf.cpp:75-130)."""

    def __init__(self, sigmaX, sigmaY, sigmaZ, nStdX, nStdY, nStdZ, params: ImageParams):
        k = _gaussian_kernel([sigmaX, sigmaY, sigmaZ], [nStdX, nStdY, nStdZ], params)
        super().__init__(k.weights)


class ConvolutionKernelGaussianMixture(ConvolutionKernel):
    """ConvolutionKernelGaussianMixture (src/operators/OperatorVarPsf.cpp:132-245)."""

    def __init__(self, sigmaX1, sigmaY1, sigmaZ1, sigmaX2, sigmaY2, sigmaZ2, weight2,
                 nStdX, nStdY, nStdZ, params: ImageParams):
        k = _gaussian_kernel([sigmaX1, sigmaY1, sigmaZ1, sigmaX2, sigmaY2, sigmaZ2, weight2],
                             [nStdX, nStdY, nStdZ], params)
        super().__init__(k.weights)


class OperatorVarPsfDevice:
    """Spatially variant image-space PSF (OperatorVarPsf / OperatorVarPsfDevice):
    OperatorVarPsfDevice(image_params) or OperatorVarPsfDevice(fname,
    image_params).  CSV: range x y z; gap x y z; nstd x y z; then one row per
    kernel with 3 sigmas (Gaussian) or 7 values (two-Gaussian mixture)."""

    def __init__(self, *args):
        self._h = None
        self._kernels = []
        self._range = None
        self._gap = None
        if len(args) == 1:
            self.params = args[0]
        elif len(args) == 2:
            self.params = args[1]
            self.readFromFile(args[0])
        else:
            raise RuntimeError("OperatorVarPsfDevice(image_params) or (fname, image_params)")

    def setRangeAndGap(self, xRange, xGap, yRange, yGap, zRange, zGap):
        self._range = np.array([xRange, yRange, zRange], np.float32)
        self._gap = np.array([xGap, yGap, zGap], np.float32)
        self._upload()

    def setKernelCollection(self, kernels):
        self._kernels = [k if isinstance(k, ConvolutionKernel) else ConvolutionKernel(k)
                         for k in kernels]
        self._upload()

    def readFromFile(self, fname: str):
        rows = []
        with open(fname) as f:
            for line in f:
                vals = [v for v in line.replace(",", " ").split() if v]
                if vals:
                    rows.append([float(v) for v in vals])
        if len(rows) <= 3:
            raise RuntimeError("CSV file format error: At least 4 rows expected")
        cols = max(len(r) for r in rows)
        if cols not in (3, 7):
            raise RuntimeError("CSV file format error: 3 columns expected for 1-Gaussian "
                               "VarPSF or 7 columns expected for 2-Gaussian VarPSF")
        rows = [r + [0.0] * (cols - len(r)) for r in rows]
        self._range = np.array(rows[0][:3], np.float32)
        self._gap = np.array(rows[1][:3], np.float32)
        nstd = rows[2][:3]
        self._kernels = [_gaussian_kernel(r[:cols], nstd, self.params) for r in rows[3:]]
        self._upload()

    def _upload(self):
        if self._range is None or not self._kernels:
            return
        w = np.concatenate([k.weights.ravel() for k in self._kernels]).astype(np.float32)
        half = np.array([k.half_sizes for k in self._kernels], np.int32).ravel()
        h = ctypes.c_void_p()
        L.check(L.lib().yrtb_varpsf_create(w.ctypes.data, half.ctypes.data,
                                           len(self._kernels), self._range.ctypes.data,
                                           self._gap.ctypes.data, ctypes.byref(h)))
        self._release()
        self._h = h

    def _release(self):
        if self._h is not None:
            L.lib().yrtb_varpsf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def _apply(self, img_in, img_out, adjoint, params=None):
        if self._h is None:
            raise RuntimeError("LUT not defined")
        for t in (img_in, img_out):
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                raise RuntimeError("images must be contiguous float32 CUDA tensors")
        if img_in.numel() != img_out.numel():
            raise RuntimeError("Dimensions mismatch between the two images")
        ip = params or self.params
        if img_in.numel() != ip.numVoxels * ip.nt:
            ip = ip.withFrames(img_in.numel() // ip.numVoxels)
        L.check(L.lib().yrtb_varpsf_apply(self._h, img_in.data_ptr(), img_out.data_ptr(),
                                          ctypes.byref(ip._c()), int(adjoint), _stream()))
        return img_out

    def applyA(self, img_in, img_out, params: Optional[ImageParams] = None):
        return self._apply(img_in, img_out, False, params)

    def applyAH(self, img_in, img_out, params: Optional[ImageParams] = None):
        return self._apply(img_in, img_out, True, params)

    @property
    def handle(self):
        return self._h
