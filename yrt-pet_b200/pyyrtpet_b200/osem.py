"""OSEM driver mirroring the reference OSEM / OSEM_GPU hooks.

Reference (paths inside yrt-pet): src/recon/OSEM.cpp:315-365 (reconstruct),
:788-811 (iterate), :926-1035 (sensitivity images, list-mode 1/numSubsets);
src/recon/OSEM_GPU.cu:311-537 (buffers, mask, EM, update);
src/recon/Corrector.cpp (which correction applies to which bin).

The list-mode loop itself runs inside libyrtb (yrtb_osem_listmode, optionally
one CUDA graph per subset); histogram mode is driven from here subset by
subset through the C ABI.  Per-event correction factors (sensitivity from a
histogram, attenuation from a mu-map or an ACF histogram, additive terms) are
computed on the device once per reconstruction.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional

import numpy as np
import torch

from . import _lib as L
from .core import (DeviceEvents, DeviceProjector, Histogram3D, ImageParams,
                   ListModeLUT, ProjectorParams, Scanner, _dev, _ptr, _stream)
from .psf import OperatorPsfDevice, OperatorVarPsfDevice
from .ranges import RangeList, iteration_filename


class OSEM_GPU:
    DEFAULT_HARD_THRESHOLD = 1.0
    DEFAULT_DENOM_THRESHOLD = 1e-35
    INITIAL_VALUE_MLEM = 0.125
    EPS_FLT = 1.19209e-07

    def __init__(self, scanner: Scanner):
        self.scanner = scanner
        self.num_MLEM_iterations = 10
        self.num_OSEM_subsets = 1
        self.hardThreshold = self.DEFAULT_HARD_THRESHOLD
        self.denomThreshold = self.DEFAULT_DENOM_THRESHOLD
        self.projectorParams = ProjectorParams(scanner)
        self.imageParams: Optional[ImageParams] = None
        self.usingListModeInput = False
        # One CUDA graph per subset, captured by every reconstruction and
        # replayed once per iteration: the capture costs more than the
        # launches it saves at a few iterations (C1, 2 x 5 subsets: 4.23 ms
        # with graphs, 3.78 ms without), so it is off by default.
        self.useGraphs = False
        # Reorder events subset-major and by LOR before iterating (GPU
        # coherence); results differ from file order only by FP summation
        # order.
        self.orderEvents = True
        # Pick the launch configuration (block size, threads per LOR, ray
        # length binning of the event order) by timing EM steps over a sample
        # of the events before reconstructing (yrtb_autotune).
        self.autotune = False
        self.lastTuneReport = None
        # Fixed launch configuration (a dict as returned by
        # DeviceProjector.get_launch, e.g. lastTuneReport["best"] of an
        # earlier reconstruction); used when autotune is off.
        self.launchConfig = None
        self._data = None
        self._sens_images: List[torch.Tensor] = []
        self._sens_histo = None
        self._invert_sens = False
        self._acf_histo = None
        self._att_image = None
        self._att_params = None
        self._randoms_histo = None
        self._scatter_histo = None
        self._global = 1.0
        self._initial = None
        self._mask = None
        self._frame_scale = None
        self.imagePsf = None
        self.flagImagePSF = False
        self.saveIterRanges = RangeList()
        self.saveIterPath = ""
        self._save_writer = None

    # ----------------------------------------------------------- setters --
    def setImageParams(self, p: ImageParams):
        self.imageParams = p

    def getImageParams(self) -> ImageParams:
        return self.imageParams

    def setDataInput(self, data):
        self._data = data
        self.usingListModeInput = isinstance(data, ListModeLUT)

    def getDataInput(self):
        return self._data

    def setSaveIterRanges(self, range_list, path: str, writer=None):
        """Save the image after the iterations in range_list (a RangeList or
        its string form, 1-based) to path with "_iterationNN" inserted before
        the extension (OSEM::setSaveIterRanges, src/recon/OSEM.cpp:651-655,
        813-821).  writer(fname, image) writes one image (a CPU float32
        array shaped like the reconstruction); by default .npy paths get
        numpy's format and any other path the raw float32 voxels (NIfTI
        writing is not part of this package: pass a writer for it)."""
        self.saveIterRanges = (range_list if isinstance(range_list, RangeList)
                               else RangeList(str(range_list)))
        self.saveIterPath = path
        self._save_writer = writer

    def _save_iteration(self, iteration: int, img: torch.Tensor, shape):
        """After MLEM iteration `iteration` (0-based): write the image when
        the iteration is in saveIterRanges (OSEM.cpp:345-348)."""
        if self.saveIterRanges.empty() or not self.saveIterRanges.isIn(iteration + 1):
            return
        fname = iteration_filename(self.saveIterPath, iteration,
                                   self.num_MLEM_iterations)
        arr = img.reshape(shape).detach().cpu().numpy()
        if self._save_writer is not None:
            self._save_writer(fname, arr)
        elif fname.endswith(".npy"):
            np.save(fname, arr)
        else:
            arr.astype(np.float32).tofile(fname)

    def setListModeEnabled(self, enabled: bool):
        self.usingListModeInput = bool(enabled)

    def isListModeEnabled(self) -> bool:
        return self.usingListModeInput

    def addTOF(self, width_ps: float, n_std: int):
        self.projectorParams.addTOF(width_ps, n_std)

    def setNumRays(self, n: int):
        self.projectorParams.numRays = int(n)

    def setProjector(self, name: str):
        self.projectorParams.setProjector(name)

    def addProjPSF(self, fname: str):
        self.projectorParams.projPsf_fname = fname

    # --------------------------------------------------- image-space PSF --
    # OSEM_GPU::addImagePSF / addUniformGaussianImagePSFFrom{FWHM,Sigma}
    # (src/recon/OSEM_GPU.cu:48-95): UNIFORM (separable, OperatorPsfDevice) or
    # VARIANT (kernel LUT, OperatorVarPsfDevice; image parameters first).
    def addImagePSF(self, image_psf_fname: str, image_psf_mode: str = "UNIFORM"):
        if not image_psf_fname:
            raise RuntimeError("Empty filename for Image-space PSF")
        mode = str(getattr(image_psf_mode, "name", image_psf_mode)).upper()
        if mode == "UNIFORM":
            self.imagePsf = OperatorPsfDevice(image_psf_fname)
        elif mode == "VARIANT":
            if self.imageParams is None:
                raise RuntimeError("For spatially variant PSF, image parameters have "
                                   "to be set before calling addImagePSF")
            self.imagePsf = OperatorVarPsfDevice(image_psf_fname,
                                                 self.imageParams.withFrames(1))
        else:
            raise RuntimeError("Unknown image PSF mode")
        self.flagImagePSF = True

    def addUniformGaussianImagePSFFromFWHM(self, fwhm_x, fwhm_y, fwhm_z,
                                           kernel_size_x=None, kernel_size_y=None,
                                           kernel_size_z=None):
        ip = self._require_image_params()
        self.imagePsf = OperatorPsfDevice.createGaussianFromFWHM(
            fwhm_x, fwhm_y, fwhm_z, ip.vx, ip.vy, ip.vz,
            kernel_size_x, kernel_size_y, kernel_size_z)
        self.flagImagePSF = True

    def addUniformGaussianImagePSFFromSigma(self, sigma_x, sigma_y, sigma_z,
                                            kernel_size_x=None, kernel_size_y=None,
                                            kernel_size_z=None):
        ip = self._require_image_params()
        self.imagePsf = OperatorPsfDevice.createGaussianFromSigma(
            sigma_x, sigma_y, sigma_z, ip.vx, ip.vy, ip.vz,
            kernel_size_x, kernel_size_y, kernel_size_z)
        self.flagImagePSF = True

    def hasImagePSF(self) -> bool:
        return self.flagImagePSF

    def _require_image_params(self) -> ImageParams:
        if self.imageParams is None:
            raise RuntimeError("Image parameters not set")
        return self.imageParams

    def setGlobalScalingFactor(self, g: float):
        self._global = float(g)

    def setSensitivityHistogram(self, h: Histogram3D):
        self._sens_histo = h

    def setInvertSensitivity(self, invert: bool = True):
        self._invert_sens = bool(invert)

    def setACFHistogram(self, h: Histogram3D):
        self._acf_histo = h

    setHardwareACFHistogram = setACFHistogram

    def setAttenuationImage(self, img, params: ImageParams):
        """mu-map in the reference's units (cm^-1 per mm path: ACF =
        exp(-0.1 * line integral))."""
        self._att_image = _dev(img, torch.float32).reshape(-1)
        self._att_params = params

    setHardwareAttenuationImage = setAttenuationImage

    def setRandomsHistogram(self, h: Histogram3D):
        self._randoms_histo = h

    def setScatterHistogram(self, h: Histogram3D):
        self._scatter_histo = h

    def setInitialEstimate(self, img):
        self._initial = _dev(img, torch.float32)

    def setMaskImage(self, img):
        self._mask = _dev(img, torch.float32).reshape(-1)

    def setFrameScaling(self, scales):
        """Per-frame sensitivity scaling c_r (updateEMThresholdDynamic with
        sensScaling)."""
        self._frame_scale = _dev(scales, torch.float32)

    def setSensitivityImages(self, imgs):
        self._sens_images = [_dev(i, torch.float32).reshape(-1) for i in imgs]

    def setSensitivityImage(self, img, subset: int = 0):
        while len(self._sens_images) <= subset:
            self._sens_images.append(None)
        self._sens_images[subset] = _dev(img, torch.float32).reshape(-1)

    def getExpectedSensImagesAmount(self) -> int:
        return 1 if self.usingListModeInput else self.num_OSEM_subsets

    # ------------------------------------------------- helper projectors --
    def _sens_projector(self) -> DeviceProjector:
        pp = ProjectorParams(self.scanner)
        pp.projectorType = self.projectorParams.projectorType
        pp.numRays = self.projectorParams.numRays
        pp.projPsf_fname = self.projectorParams.projPsf_fname
        pp._psf = self.projectorParams._psf
        pp.precision = self.projectorParams.precision
        # Compensated precision accumulates the sensitivity image exactly
        # (64-bit fixed point, the deterministic two-pass back projection):
        # it sums every histogram bin's contribution once per reconstruction.
        pp.deterministic = (self.projectorParams.deterministic or
                            self.projectorParams.precision == L.YRTB_COMPENSATED)
        return DeviceProjector(self.scanner, self.imageParams.withFrames(1), pp)

    def _histo_dev(self, h):
        if h is None:
            return None
        if getattr(h, "data", None) is None:
            return None
        return _dev(h.data, torch.float32)

    # ----------------------------------------------- sensitivity images --
    def generateSensitivityImages(self) -> List[torch.Tensor]:
        """Back projection of sens x ACF over every Histogram3D bin (non-TOF);
        with an image-space PSF, PSF^H of it zeroed where the back projection
        is <= EPS_FLT (OSEM_GPU.cu:228-236); then thresholded: <= hardThreshold
        -> 0, else x globalScale."""
        if self.imageParams is None:
            raise RuntimeError("Image parameters not valid/set")
        nsub = 1 if self.usingListModeInput else self.num_OSEM_subsets
        proj = self._sens_projector()
        sh = self._histo_dev(self._sens_histo)
        if sh is not None and self._invert_sens:
            sh = torch.where(sh != 0, 1.0 / sh, sh)
        acf = self._histo_dev(self._acf_histo)
        ip = self.imageParams
        out = []
        for s in range(nsub):
            img = torch.zeros(ip.numVoxels, dtype=torch.float32, device="cuda")
            proj.sensitivity_histo3d(img, nsub, s, sens_histo=sh, acf_histo=acf,
                                     mu=None if acf is not None else self._att_image,
                                     mu_params=self._att_params)
            if self.flagImagePSF:
                blurred = torch.empty_like(img)
                self.imagePsf.applyAH(img, blurred, ip.withFrames(1))
                L.check(L.lib().yrtb_apply_threshold(
                    blurred.data_ptr(), img.data_ptr(), ip.numVoxels, 1, 0,
                    float(self.EPS_FLT), 0.0, 0.0, 1.0, 0.0, _stream()))
                img = blurred
            L.check(L.lib().yrtb_apply_threshold(
                img.data_ptr(), img.data_ptr(), ip.numVoxels, 1, 0,
                float(self.hardThreshold), 0.0, 0.0, float(self._global), 0.0,
                _stream()))
            out.append(img)
        self._sens_images = out
        return out

    # ------------------------------------------------------- reconstruct --
    def _listmode_events(self, proj: DeviceProjector, lm: ListModeLUT,
                         order_subsets: int = 0):
        """Device events with their correction factors.  With order_subsets,
        the events are first put in subset-major order (yrtb_events_subset_
        order) and the corrections are computed on the ordered arrays, so
        that the attenuation walks also run on grouped rays; returns
        (events, subset offsets or None)."""
        base = lm.device_events()
        ev = DeviceEvents(base.count, base.d1, base.d2, base.lor, base.tof,
                          base.frame, base.motion_frame, base.motion)
        if lm.randoms is not None:
            ev.additive = base.additive if base.additive is not None else _dev(
                lm.randoms, torch.float32)
        offsets = None
        if self.launchConfig is not None and not self.autotune:
            proj.set_launch(**self.launchConfig)
        if self.autotune:
            probe = torch.full(proj.img_params.shape, self.INITIAL_VALUE_MLEM,
                               dtype=torch.float32, device="cuda")
            self.lastTuneReport = proj.autotune(probe, ev, max(order_subsets, 1))
            del probe
        if order_subsets:
            ev, offsets = proj.order_events(ev, order_subsets)
        if self._sens_histo is not None:
            sh = self._histo_dev(self._sens_histo)
            ev.sens = proj.gather_histo3d(sh, ev, invert=self._invert_sens)
        if self._acf_histo is not None:
            ev.att = proj.gather_histo3d(self._histo_dev(self._acf_histo), ev)
        elif self._att_image is not None:
            ev.att = proj.attenuation_factors(self._att_image, self._att_params,
                                              ev)
        add = ev.additive
        if add is None and self._randoms_histo is not None:
            add = proj.gather_histo3d(self._histo_dev(self._randoms_histo), ev)
        if self._scatter_histo is not None:
            sc = proj.gather_histo3d(self._histo_dev(self._scatter_histo), ev)
            add = sc if add is None else add + sc
        ev.additive = add
        if proj.take_event_errors():
            raise RuntimeError("A Line-Of-Response might not respect the "
                               "Minimum-Angle-Difference restriction of the "
                               "scanner (or a detector id is out of range)")
        return ev, offsets

    def reconstruct(self, out_fname: str = "") -> torch.Tensor:
        if self._data is None:
            raise RuntimeError("Data input unspecified")
        if not self._sens_images:
            raise RuntimeError("Sensitivity image(s) not set")
        if self.num_OSEM_subsets <= 0 or self.num_MLEM_iterations <= 0:
            raise RuntimeError("Not enough OSEM subsets / MLEM iterations")
        if self.imageParams is None:
            raise RuntimeError("Image parameters not valid/set")
        if len(self._sens_images) != self.getExpectedSensImagesAmount():
            raise RuntimeError(
                "The number of sensitivity images provided does not match the "
                f"number of subsets. Expected {self.getExpectedSensImagesAmount()}"
                f" but received {len(self._sens_images)}")
        if self.usingListModeInput:
            return self._reconstruct_listmode()
        return self._reconstruct_histogram()

    def _reconstruct_listmode(self) -> torch.Tensor:
        lm: ListModeLUT = self._data
        nt = lm.getNumDynamicFrames()
        ip = self.imageParams.withFrames(nt)
        proj = DeviceProjector(self.scanner, ip, self.projectorParams)
        ev, offsets = self._listmode_events(
            proj, lm, self.num_OSEM_subsets if self.orderEvents else 0)
        if self.projectorParams.numRays > 1:
            # Multi-ray offsets of every item index a subset call uses, drawn
            # once for the whole reconstruction.
            S = self.num_OSEM_subsets
            proj.multiray_table((ev.count + S - 1) // S)
        J = ip.numVoxels
        img = torch.empty(nt * J, dtype=torch.float32, device="cuda")
        init = 0
        if self._initial is not None:
            img.copy_(self._initial.reshape(-1))
            init = 1
        psf = self.imagePsf if self.flagImagePSF else None
        work = torch.empty((3 * nt + 1) * J if psf else nt * J + J,
                           dtype=torch.float32, device="cuda")
        sens = self._sens_images[0]
        if self._mask is not None:
            mask_src = self._mask
        else:
            mask_src = sens
        # yrtb_osem_listmode masks with its sensitivity argument; give it the mask
        # first when a separate mask image is set.
        p = L.yrtb_osem_params(self.num_MLEM_iterations, self.num_OSEM_subsets,
                               self._global, self.denomThreshold, self.EPS_FLT,
                               init, int(self.useGraphs),
                               _ptr(self._frame_scale),
                               None if offsets is None else offsets.ctypes.data,
                               None if not isinstance(psf, OperatorPsfDevice) else psf.handle,
                               None if not isinstance(psf, OperatorVarPsfDevice) else psf.handle)
        stream = torch.cuda.current_stream()
        use_side = self.useGraphs and stream.cuda_stream == 0
        s = torch.cuda.Stream() if use_side else stream
        if use_side:
            s.wait_stream(stream)
        with torch.cuda.stream(s):
            if mask_src is not sens:
                if not init:
                    L.check(L.lib().yrtb_fill(img.data_ptr(), img.numel(),
                                              self.INITIAL_VALUE_MLEM,
                                              _stream()))
                L.check(L.lib().yrtb_apply_threshold(
                    img.data_ptr(), mask_src.data_ptr(), J, nt, 1, 0.0, 0.0,
                    0.0, 1.0, 0.0, _stream()))
                p.init_from_image = 1
            if self.saveIterRanges.empty():
                L.check(L.lib().yrtb_osem_listmode(proj.h, ctypes.byref(ev.c()),
                                                   sens.data_ptr(), img.data_ptr(),
                                                   work.data_ptr(), ctypes.byref(p),
                                                   _stream()))
            else:
                # One call per iteration, each continuing from the image of
                # the last (the same passes: the mask is idempotent and the
                # subset sensitivity is rebuilt the same way), so that the
                # chosen iterations can be saved.
                p.iterations = 1
                for it in range(self.num_MLEM_iterations):
                    L.check(L.lib().yrtb_osem_listmode(proj.h, ctypes.byref(ev.c()),
                                                       sens.data_ptr(), img.data_ptr(),
                                                       work.data_ptr(), ctypes.byref(p),
                                                       _stream()))
                    p.init_from_image = 1
                    self._save_iteration(it, img, ip.shape)
        if use_side:
            stream.wait_stream(s)
        self._last_events = ev
        return img.reshape(ip.shape)

    def _reconstruct_histogram(self) -> torch.Tensor:
        h: Histogram3D = self._data
        ip = self.imageParams.withFrames(1)
        proj = DeviceProjector(self.scanner, ip, self.projectorParams)
        J = ip.numVoxels
        meas = _dev(h.data, torch.float32)
        sh = self._histo_dev(self._sens_histo)
        if sh is not None and self._invert_sens:
            sh = torch.where(sh != 0, 1.0 / sh, sh)
        acf = self._histo_dev(self._acf_histo)
        add = self._histo_dev(self._randoms_histo)
        sc = self._histo_dev(self._scatter_histo)
        if sc is not None:
            add = sc if add is None else add + sc
        img = torch.empty(J, dtype=torch.float32, device="cuda")
        if self._initial is not None:
            img.copy_(self._initial.reshape(-1))
        else:
            img.fill_(self.INITIAL_VALUE_MLEM)
        if self._mask is not None:
            mask = self._mask
        elif self.num_OSEM_subsets == 1:
            mask = self._sens_images[0]
        else:
            mask = torch.stack(self._sens_images).sum(0)
        L.check(L.lib().yrtb_apply_threshold(img.data_ptr(), mask.data_ptr(), J,
                                             1, 1, 0.0, 0.0, 0.0, 1.0, 0.0,
                                             _stream()))
        em = torch.empty(J, dtype=torch.float32, device="cuda")
        # The bins each subset's EM pass does work for (valid pair, non-zero
        # measurement), selected once per reconstruction: the passes then
        # run full warps of such bins instead of skipping empty bins inside
        # each warp.
        S = self.num_OSEM_subsets
        bins = []
        for s in range(S):
            nps = h.numPhi // S + (1 if s + (h.numPhi // S) * S < h.numPhi else 0)
            bins.append(proj.histo3d_subset_nonzero(meas, S, s,
                                                    h.numR * nps * h.numZBin))
        psf = self.imagePsf if self.flagImagePSF else None
        if psf is not None:
            # Project PSF x, apply PSF^H to the EM image
            # (OSEM_GPU::computeEMUpdateImage, OSEM_GPU.cu:456-509).
            xpsf = torch.empty_like(img)
            em_psf = torch.empty_like(em)
        for it in range(self.num_MLEM_iterations):
            for s in range(self.num_OSEM_subsets):
                em.zero_()
                if psf is not None:
                    psf.applyA(img, xpsf, ip)
                proj.em_step_histo3d(img if psf is None else xpsf, em, meas,
                                     self.num_OSEM_subsets, s,
                                     sens_histo=sh, acf_histo=acf,
                                     additive_histo=add,
                                     global_scale=self._global,
                                     denom_threshold=self.denomThreshold,
                                     bins=bins[s])
                if psf is not None:
                    psf.applyAH(em, em_psf, ip)
                L.check(L.lib().yrtb_em_update(
                    img.data_ptr(), (em if psf is None else em_psf).data_ptr(),
                    self._sens_images[s].data_ptr(), J, 1, 1, self.EPS_FLT,
                    None, _stream()))
            self._save_iteration(it, img, ip.shape)
        return img.reshape(ip.shape)


def createOSEM(scanner: Scanner, useGPU: bool = True, isLowRank: bool = False):
    if not useGPU:
        raise RuntimeError("pyyrtpet_b200 provides the GPU reconstruction only")
    if isLowRank:
        from .lrem import LREM_GPU
        return LREM_GPU(scanner)
    return OSEM_GPU(scanner)
