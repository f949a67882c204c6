"""Host-side mirror of YRT-PET's projector / OSEM Python surface over libyrtb.

Class and method names follow the reference's pybind11 module and its
``pyyrtpet.ProjectionOper`` wrapper so that reference scripts port by
changing the import.  Images are torch tensors (float32, shape
``(nt, nz, ny, nx)``) on the CUDA device; projection data are numpy or torch
arrays.  torch is used for device memory and streams only; every projection
runs in libyrtb's CUDA kernels and there is no CPU fallback.

Reference surfaces mirrored (paths inside yrt-pet):
  Scanner                   src/datastruct/scanner/Scanner.cpp:102-183
  ImageParams               src/datastruct/image/ImageParams.cpp:136-218
  ProjectorParams           include/yrt-pet/operators/ProjectorParams.hpp:27-71
  ListModeLUT               include/yrt-pet/datastruct/projection/ListModeLUT.hpp
  Histogram3D, BinIterators src/datastruct/projection/Histogram3D.cpp,
                            src/datastruct/projection/BinIterator.cpp
  OperatorProjectorDevice   src/operators/OperatorProjectorDevice.cu:26-90
  ProjectionOper            python/pyyrtpet/_pyyrtpet.py:81-157
  OSEM / createOSEM         src/recon/OSEM.cpp:36-162, src/utils/ReconstructionUtils.cpp:915-933
  convertToHistogram3D      src/utils/ReconstructionUtils.cpp:659-800
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib as L

# ------------------------------------------------------------------ helpers --


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    return t.data_ptr()


def _dev(a, dtype, device="cuda"):
    """numpy / torch array -> contiguous CUDA tensor of the given torch dtype."""
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        t = a
    else:
        arr = np.ascontiguousarray(a)
        if arr.dtype == np.uint32:
            arr = arr.view(np.int32)
        t = torch.from_numpy(arr)
    if t.dtype != dtype:
        if dtype == torch.int32 and t.dtype == torch.uint32:
            t = t.view(torch.int32)
        else:
            t = t.to(dtype)
    return t.to(device, non_blocking=True).contiguous()


# ------------------------------------------------------------------ Scanner --
class Scanner:
    """Cylindrical scanner with a regular detector LUT (DetRegular)."""

    def __init__(self, scannerName: str, axialFOV: float, crystalSize_z: float,
                 crystalSize_trans: float, crystalDepth: float,
                 scannerRadius: float, detsPerRing: int, numRings: int,
                 numDOI: int = 1, maxRingDiff: int = 0, minAngDiff: int = 1,
                 detsPerBlock: int = 1):
        self.scannerName = scannerName
        self.axialFOV = float(axialFOV)
        self.crystalSize_z = float(crystalSize_z)
        self.crystalSize_trans = float(crystalSize_trans)
        self.crystalDepth = float(crystalDepth)
        self.scannerRadius = float(scannerRadius)
        self.detsPerRing = int(detsPerRing)
        self.numRings = int(numRings)
        self.numDOI = int(numDOI)
        self.maxRingDiff = int(maxRingDiff)
        self.minAngDiff = int(minAngDiff)
        self.detsPerBlock = int(detsPerBlock)
        if self.maxRingDiff >= self.numRings:
            raise RuntimeError("Maximum Ring difference has to be lower than "
                               "the number of rings")
        if self.minAngDiff <= 0:
            raise RuntimeError("Minimum angle difference has to be non-zero")
        self._lut = None
        self._custom_lut = None

    def _c(self) -> L.yrtb_scanner:
        return L.yrtb_scanner(self.axialFOV, self.crystalSize_z,
                              self.crystalSize_trans, self.crystalDepth,
                              self.scannerRadius, self.detsPerRing,
                              self.numRings, self.numDOI, self.maxRingDiff,
                              self.minAngDiff, self.detsPerBlock)

    def getNumDets(self) -> int:
        return self.detsPerRing * self.numRings * self.numDOI

    def getExpectedNumDets(self) -> int:
        return self.getNumDets()

    def createLUT(self) -> np.ndarray:
        """(numDets, 6) float32: x, y, z, orient x, y, z."""
        if self._custom_lut is not None:
            return self._custom_lut
        if self._lut is None:
            out = np.zeros((self.getNumDets(), 6), np.float32)
            L.check(L.lib().yrtb_scanner_regular_lut(
                ctypes.byref(self._c()), out.ctypes.data))
            self._lut = out
        return self._lut

    def setDetectorLUT(self, lut: np.ndarray):
        """Arbitrary crystal positions/orientations (DetCoord)."""
        lut = np.ascontiguousarray(lut, np.float32).reshape(-1, 6)
        if lut.shape[0] != self.getNumDets():
            raise RuntimeError("The number of detectors given by the LUT does "
                               "not match the scanner's characteristics")
        self._custom_lut = lut

    def getDetectorPos(self, d: int):
        return tuple(float(v) for v in self.createLUT()[d, :3])

    def getDetectorOrient(self, d: int):
        return tuple(float(v) for v in self.createLUT()[d, 3:])


# -------------------------------------------------------------- ImageParams --
class ImageParams:
    def __init__(self, nx: int, ny: int, nz: int, length_x: float,
                 length_y: float, length_z: float, off_x: float = 0.0,
                 off_y: float = 0.0, off_z: float = 0.0, nt: int = 1):
        self.nx, self.ny, self.nz, self.nt = int(nx), int(ny), int(nz), int(nt)
        if min(self.nx, self.ny, self.nz, self.nt) <= 0:
            raise RuntimeError("ImageParams object incomplete")
        self.length_x = float(length_x)
        self.length_y = float(length_y)
        self.length_z = float(length_z)
        self.off_x, self.off_y, self.off_z = float(off_x), float(off_y), float(off_z)
        f32 = np.float32
        self.vx = float(f32(self.length_x) / f32(self.nx))
        self.vy = float(f32(self.length_y) / f32(self.ny))
        self.vz = float(f32(self.length_z) / f32(self.nz))
        fr = max(f32(self.length_x) / f32(2), f32(self.length_y) / f32(2))
        self.fovRadius = float(f32(fr) - max(f32(self.vx), f32(self.vy)) / f32(1000))

    @staticmethod
    def fromParams(nx, ny, nz, vx, vy, vz, nt=1):
        return ImageParams(nx, ny, nz, nx * vx, ny * vy, nz * vz, nt=nt)

    def _c(self) -> L.yrtb_image_params:
        return L.yrtb_image_params(self.nx, self.ny, self.nz, self.nt,
                                   self.length_x, self.length_y, self.length_z,
                                   self.off_x, self.off_y, self.off_z)

    @property
    def shape(self):
        return (self.nt, self.nz, self.ny, self.nx)

    @property
    def numVoxels(self) -> int:
        return self.nx * self.ny * self.nz

    def isSameAsIgnoreFrames(self, o: "ImageParams") -> bool:
        return ((self.nx, self.ny, self.nz) == (o.nx, o.ny, o.nz) and
                abs(self.length_x - o.length_x) < 1e-4 and
                abs(self.length_y - o.length_y) < 1e-4 and
                abs(self.length_z - o.length_z) < 1e-4)

    def withFrames(self, nt: int) -> "ImageParams":
        return ImageParams(self.nx, self.ny, self.nz, self.length_x,
                           self.length_y, self.length_z, self.off_x,
                           self.off_y, self.off_z, nt)


# ---------------------------------------------------------- ProjectorParams --
def read_psf_csv(fname: str):
    """Projection-space PSF table in ProjectionPsfManager's CSV format
    (ProjectionPsfManager.cpp:27-50): sStep, kSpacing, kernelSize, then
    numS * kernelSize taps, all on the first row."""
    with open(fname) as f:
        vals = [float(v) for v in f.read().replace("\n", ",").split(",")
                if v.strip()]
    s_step, k_spacing, size = vals[0], vals[1], int(vals[2])
    if size % 2 == 0:
        raise RuntimeError("Kernels must be of odd length")
    taps = np.asarray(vals[3:], np.float32)
    num_s = len(taps) // size
    return s_step, k_spacing, taps[:num_s * size].reshape(num_s, size)


def write_psf_csv(fname: str, s_step: float, k_spacing: float, taps):
    taps = np.asarray(taps, np.float32).reshape(-1, np.shape(taps)[-1])
    row = [repr(float(s_step)), repr(float(k_spacing)), str(taps.shape[1])]
    row += [repr(float(v)) for v in taps.ravel()]
    with open(fname, "w") as f:
        f.write(",".join(row) + "\n")


class ProjectorParams:
    def __init__(self, scanner: Scanner):
        self.scanner = scanner
        self.projectorType = "S"
        self.numRays = 1
        self.projPsf_fname = ""
        self.updaterType = "DEFAULT4D"
        # Low-rank updater: HBasis (rank x frames float32) and whether a back
        # projection accumulates onto H instead of W.
        self.HBasis = None
        self.updateH = False
        self.precision = L.YRTB_MIRROR
        # Two-pass fixed-point back projection (order-independent results).
        self.deterministic = False
        self._tofWidth_ps = 0.0
        self._tofNumStd = 0
        self._psf = None

    def setProjector(self, name: str):
        n = name.upper()
        if n in ("S", "SIDDON"):
            self.projectorType = "S"
        elif n in ("D", "DD", "DISTANCEDRIVEN", "DISTANCE_DRIVEN"):
            self.projectorType = "DD"
        else:
            raise RuntimeError(f"Unknown projector: {name}")

    def setHBasisFromNumpy(self, HBasis):
        h = np.asarray(HBasis)
        if h.ndim != 2:
            raise RuntimeError("HBasis must be 2D (rank x time).")
        if h.dtype != np.float32:
            raise RuntimeError("HBasis must be float32.")
        self.HBasis = np.ascontiguousarray(h)

    def addTOF(self, tofWidth_ps: float, tofNumStd: int):
        self._tofWidth_ps = float(tofWidth_ps)
        self._tofNumStd = int(tofNumStd)

    def removeTOF(self):
        self._tofWidth_ps = 0.0
        self._tofNumStd = 0

    def hasTOF(self) -> bool:
        return self._tofWidth_ps > 0

    def getTOFWidth_ps(self) -> float:
        return self._tofWidth_ps

    def getTOFNumStd(self) -> int:
        return self._tofNumStd

    def setProjPsf(self, s_step, k_spacing, taps):
        self._psf = (float(s_step), float(k_spacing),
                     np.ascontiguousarray(taps, np.float32))

    def _psf_table(self):
        if self._psf is not None:
            return self._psf
        if self.projPsf_fname:
            return read_psf_csv(self.projPsf_fname)
        return None

    def _c(self):
        psf = self._psf_table() if self.projectorType == "DD" else None
        keep = None
        p = L.yrtb_projector_params(
            L.YRTB_SIDDON if self.projectorType == "S" else L.YRTB_DD,
            int(self.numRays), self._tofWidth_ps, self._tofNumStd, 0, 0, 0.0,
            0.0, None, int(self.precision), int(bool(self.deterministic)))
        if psf is not None:
            s_step, k_spacing, taps = psf
            keep = np.ascontiguousarray(taps, np.float32)
            p.psf_num_s, p.psf_size = keep.shape
            p.psf_s_step, p.psf_k_spacing = s_step, k_spacing
            p.psf_taps = keep.ctypes.data
        return p, keep


# ------------------------------------------------------------- bin iterators --
@dataclass
class BinIteratorChronologicalInterleaved:
    """Events idx, idx+S, idx+2S, ... (BinIterator.cpp:261-265)."""
    numSubsets: int
    numEvents: int
    idxSubset: int

    def size(self) -> int:
        if self.numEvents <= self.idxSubset:
            return 0
        return (self.numEvents - 1 - self.idxSubset) // self.numSubsets + 1

    def get(self, i: int) -> int:
        return self.idxSubset + self.numSubsets * i

    def indices(self) -> np.ndarray:
        return np.arange(self.idxSubset, self.numEvents, self.numSubsets,
                         dtype=np.int64)

    def _range(self) -> L.yrtb_range:
        return L.yrtb_range(self.idxSubset, self.numSubsets, 0)


@dataclass
class BinIteratorRangeHistogram3D:
    """Bins with phi = idx mod S, all r and z (BinIterator.cpp:147-198)."""
    numZBin: int
    numPhi: int
    numR: int
    numSubsets: int
    idxSubset: int

    def __post_init__(self):
        self.numPhiSubset = self.numPhi // self.numSubsets
        if self.idxSubset + self.numPhiSubset * self.numSubsets < self.numPhi:
            self.numPhiSubset += 1

    def size(self) -> int:
        return self.numR * self.numPhiSubset * self.numZBin

    def indices(self) -> np.ndarray:
        idx = np.arange(self.size(), dtype=np.int64)
        per = self.numPhiSubset * self.numR
        z = idx // per
        phi = (idx % per) // self.numR * self.numSubsets + self.idxSubset
        r = (idx % per) % self.numR
        return z * self.numPhi * self.numR + phi * self.numR + r


# ---------------------------------------------------------- projection data --
class ProjectionData:
    """Common base: the reference ProjectionData interface used here."""
    scanner: Scanner

    def getScanner(self) -> Scanner:
        return self.scanner


class ListModeLUT(ProjectionData):
    """List-mode events as detector pairs (+ optional TOF, randoms,
    dynamic frames and per-event rigid motion)."""

    def __init__(self, scanner: Scanner, flagTOF: bool = False,
                 flagRandoms: bool = False):
        self.scanner = scanner
        self.flagTOF = bool(flagTOF)
        self.flagRandoms = bool(flagRandoms)
        self.d1 = np.zeros(0, np.uint32)
        self.d2 = np.zeros(0, np.uint32)
        self.tof = None
        self.randoms = None
        self.timestamps = None
        self.dynamicFrames = None
        self.motionFrames = None
        self.motionTransforms = None
        self._dev = None

    # -- construction
    def allocate(self, n: int):
        self.d1 = np.zeros(n, np.uint32)
        self.d2 = np.zeros(n, np.uint32)
        self.timestamps = np.zeros(n, np.uint32)
        if self.flagTOF:
            self.tof = np.zeros(n, np.float32)
        if self.flagRandoms:
            self.randoms = np.zeros(n, np.float32)
        self._dev = None

    def bind(self, d1, d2, tof=None, randoms=None, timestamps=None):
        """Bulk binding of event arrays (ListModeLUTAlias::bind)."""
        self.d1 = np.ascontiguousarray(d1, np.uint32)
        self.d2 = np.ascontiguousarray(d2, np.uint32)
        if len(self.d1) != len(self.d2):
            raise RuntimeError("d1 and d2 must have the same length")
        self.tof = None if tof is None else np.ascontiguousarray(tof, np.float32)
        self.flagTOF = self.tof is not None
        self.randoms = (None if randoms is None else
                        np.ascontiguousarray(randoms, np.float32))
        self.flagRandoms = self.randoms is not None
        self.timestamps = (None if timestamps is None else
                           np.ascontiguousarray(timestamps, np.uint32))
        self._dev = None

    def setDetectorIdsOfEvent(self, i, d1, d2):
        self.d1[i] = d1
        self.d2[i] = d2
        self._dev = None

    def setTOFValueOfEvent(self, i, v):
        self.tof[i] = v
        self._dev = None

    def setRandomsEstimateOfEvent(self, i, v):
        self.randoms[i] = v
        self._dev = None

    # -- file I/O (ListModeLUT format: u32 ts, u32 d1, u32 d2, [f32 tof],
    #    [f32 randoms] per event; ListModeLUT.cpp:224-307)
    def _fields(self):
        return 3 + int(self.flagTOF) + int(self.flagRandoms)

    def readFromFile(self, fname: str, device: bool = True):
        """Loads a list-mode file.  device=True: the raw bytes go to the GPU
        in one copy and are unpacked there (yrtb_unpack_listmode); the host
        arrays are filled from the device result."""
        raw = np.fromfile(fname, dtype=np.uint32)
        f = self._fields()
        if raw.size == 0 or raw.size % f != 0:
            raise RuntimeError("Error: Input file has incorrect size in "
                               "ListModeLUTOwned::readFromFile.")
        n = raw.size // f
        if device:
            d_raw = torch.from_numpy(raw.view(np.int32)).cuda()
            ts = torch.empty(n, dtype=torch.int32, device="cuda")
            d1 = torch.empty_like(ts)
            d2 = torch.empty_like(ts)
            tof = torch.empty(n, dtype=torch.float32, device="cuda") if self.flagTOF else None
            rnd = torch.empty(n, dtype=torch.float32, device="cuda") if self.flagRandoms else None
            L.check(L.lib().yrtb_unpack_listmode(
                d_raw.data_ptr(), n, int(self.flagTOF), int(self.flagRandoms),
                self.scanner.getNumDets(), ts.data_ptr(), d1.data_ptr(),
                d2.data_ptr(), _ptr(tof), _ptr(rnd), _stream()))
            self.d1 = d1.cpu().numpy().view(np.uint32)
            self.d2 = d2.cpu().numpy().view(np.uint32)
            self.timestamps = ts.cpu().numpy().view(np.uint32)
            self.tof = None if tof is None else tof.cpu().numpy()
            self.randoms = None if rnd is None else rnd.cpu().numpy()
            self._dev = DeviceEvents(n, d1, d2, tof=tof, additive=rnd)
            return self
        rec = raw.reshape(n, f)
        if np.any(rec[:, 1:3] >= self.scanner.getNumDets()):
            bad = int(np.nonzero(np.any(rec[:, 1:3] >= self.scanner.getNumDets(), axis=1))[0][0])
            raise RuntimeError(f"Detectors invalid in list-mode event {bad}")
        self.timestamps = rec[:, 0].copy()
        self.d1 = rec[:, 1].copy()
        self.d2 = rec[:, 2].copy()
        k = 3
        self.tof = None
        self.randoms = None
        if self.flagTOF:
            self.tof = rec[:, k].copy().view(np.float32)
            k += 1
        if self.flagRandoms:
            self.randoms = rec[:, k].copy().view(np.float32)
        self._dev = None
        return self

    def writeToFile(self, fname: str):
        n = self.count()
        cols = [self.timestamps if self.timestamps is not None else
                np.zeros(n, np.uint32), self.d1, self.d2]
        if self.flagTOF:
            cols.append(np.asarray(self.tof, np.float32).view(np.uint32))
        if self.flagRandoms:
            cols.append(np.asarray(self.randoms, np.float32).view(np.uint32))
        np.stack([np.asarray(c, np.uint32) for c in cols], 1).tofile(fname)

    # -- queries
    def count(self) -> int:
        return len(self.d1)

    def isUniform(self) -> bool:
        return True

    def hasTOF(self) -> bool:
        return self.tof is not None

    def hasRandomsEstimates(self) -> bool:
        return self.randoms is not None

    def getDetector1(self, i):
        return int(self.d1[i])

    def getDetector2(self, i):
        return int(self.d2[i])

    def getTOFValue(self, i):
        return float(self.tof[i])

    def getBinIter(self, numSubsets: int, idxSubset: int):
        if idxSubset < 0 or numSubsets <= 0 or idxSubset >= numSubsets:
            raise RuntimeError("The subset index has to be smaller than the "
                               "number of subsets")
        return BinIteratorChronologicalInterleaved(numSubsets, self.count(),
                                                   idxSubset)

    # -- dynamic framing and motion (ListMode.cpp:89-182)
    def addDynamicFraming(self, frame_timestamps):
        """Contiguous frames given by numFrames+1 timestamps (the reference's
        DynamicFraming vector): frame f = [ts_f, ts_{f+1}); events before the
        first or at/after the last timestamp get frame -1 (skipped).  Events
        are chronological, as ListMode::addDynamicFraming assumes
        (ListMode.cpp:137-182)."""
        if self.timestamps is None:
            raise RuntimeError("dynamic framing needs event timestamps")
        b = np.asarray(frame_timestamps, np.int64)
        if len(b) < 2:
            raise RuntimeError("Number of frames cannot be zero.")
        ts = self.timestamps.astype(np.int64)
        n = len(ts)
        fr = np.full(n, -1, np.int32)
        ev = 0
        while ev < n and ts[ev] < b[0]:
            ev += 1
        for f in range(len(b) - 1):
            e1 = ev + int(np.searchsorted(ts[ev:], b[f + 1], side="left"))
            fr[ev:e1] = f
            ev = e1
        self.dynamicFrames = fr
        self._numDynamicFrames = len(b) - 1
        self._dev = None

    def setDynamicFrames(self, frames):
        self.dynamicFrames = np.ascontiguousarray(frames, np.int32)
        self._dev = None

    def getNumDynamicFrames(self) -> int:
        if self.dynamicFrames is None:
            return 1
        n = getattr(self, "_numDynamicFrames", None)
        if n is not None:
            return n
        return int(self.dynamicFrames.max()) + 1 if len(self.dynamicFrames) else 1

    def addLORMotion(self, frame_starts, transforms):
        """Rigid motion (LORMotion): motion frame f starts at frame_starts[f]
        and lasts until the next start (the last frame until the end);
        events before the first start get frame -1 (unmoved).  transforms:
        (numFrames, 12) in transform_t order (r00 r01 r02 tx r10 r11 r12 ty
        r20 r21 r22 tz), ListMode::addLORMotion (ListMode.cpp:89-127)."""
        if self.timestamps is None:
            raise RuntimeError("LOR motion needs event timestamps")
        starts = np.asarray(frame_starts, np.int64)
        ts = self.timestamps.astype(np.int64)
        mf = np.searchsorted(starts, ts, side="right").astype(np.int32) - 1
        self.motionFrames = mf
        self.motionTransforms = np.ascontiguousarray(transforms,
                                                     np.float32).reshape(-1, 12)
        self._dev = None

    def setMotion(self, motion_frames, transforms):
        self.motionFrames = np.ascontiguousarray(motion_frames, np.int32)
        self.motionTransforms = np.ascontiguousarray(transforms,
                                                     np.float32).reshape(-1, 12)
        self._dev = None

    # -- device copy
    def device_events(self) -> "DeviceEvents":
        if self._dev is None:
            self._dev = DeviceEvents.from_listmode(self)
        return self._dev


class Histogram3D(ProjectionData):
    """Fully 3D span-1 histogram with the reference's bin layout."""

    def __init__(self, scanner: Scanner, data=None):
        if scanner.detsPerRing % 2 != 0:
            raise RuntimeError("Limitation: The number of detectors per ring "
                               "has to be even for the histogram to be "
                               "properly defined")
        self.scanner = scanner
        dims = np.zeros(3, np.uint64)
        L.check(L.lib().yrtb_histo3d_dims(ctypes.byref(scanner._c()),
                                          dims.ctypes.data))
        self.numZBin, self.numPhi, self.numR = (int(x) for x in dims)
        self.histoSize = self.numZBin * self.numPhi * self.numR
        self.data = None if data is None else np.ascontiguousarray(
            data, np.float32).reshape(-1)

    def allocate(self):
        self.data = np.zeros(self.histoSize, np.float32)

    def count(self) -> int:
        return self.histoSize

    def isUniform(self) -> bool:
        return False

    def getBinIter(self, numSubsets: int, idxSubset: int):
        if idxSubset < 0 or numSubsets <= 0 or idxSubset >= numSubsets:
            raise RuntimeError("The subset index has to be smaller than the "
                               "number of subsets")
        return BinIteratorRangeHistogram3D(self.numZBin, self.numPhi,
                                           self.numR, numSubsets, idxSubset)

    def getProjectionValue(self, b):
        return float(self.data[b])

    def getBinIdFromDetPair(self, d1, d2) -> np.ndarray:
        return histo3d_bins(self.scanner, d1, d2)

    def getDetPairFromBinId(self, bins):
        return histo3d_detpairs(self.scanner, bins)


class UniformHistogram(Histogram3D):
    def __init__(self, scanner: Scanner, value: float = 1.0):
        super().__init__(scanner)
        self.value = float(value)

    def isUniform(self) -> bool:
        return True


# ------------------------------------------------------------ device events --
@dataclass
class DeviceEvents:
    """Structure-of-arrays events resident on the GPU (yrtb_events)."""
    count: int
    d1: Optional[torch.Tensor] = None
    d2: Optional[torch.Tensor] = None
    lor: Optional[torch.Tensor] = None
    tof: Optional[torch.Tensor] = None
    frame: Optional[torch.Tensor] = None
    motion_frame: Optional[torch.Tensor] = None
    motion: Optional[torch.Tensor] = None
    measurement: Optional[torch.Tensor] = None
    sens: Optional[torch.Tensor] = None
    att: Optional[torch.Tensor] = None
    additive: Optional[torch.Tensor] = None
    perm: Optional[torch.Tensor] = None
    orient: Optional[torch.Tensor] = None
    _c_cache: object = field(default=None, repr=False)

    @staticmethod
    def from_arrays(d1=None, d2=None, *, lor=None, tof=None, frame=None,
                    motion_frame=None, motion=None, measurement=None,
                    sens=None, att=None, additive=None, orient=None,
                    device="cuda"):
        """orient (with lor): crystal orientations n1, n2, 6 floats per
        event, for distance-driven and multi-ray projection."""
        n = len(d1) if d1 is not None else len(lor)
        return DeviceEvents(
            n, _dev(d1, torch.int32, device), _dev(d2, torch.int32, device),
            _dev(lor, torch.float32, device), _dev(tof, torch.float32, device),
            _dev(frame, torch.int32, device),
            _dev(motion_frame, torch.int32, device),
            _dev(motion, torch.float32, device),
            _dev(measurement, torch.float32, device),
            _dev(sens, torch.float32, device), _dev(att, torch.float32, device),
            _dev(additive, torch.float32, device),
            orient=_dev(orient, torch.float32, device))

    @staticmethod
    def from_listmode(lm: ListModeLUT) -> "DeviceEvents":
        return DeviceEvents.from_arrays(
            lm.d1, lm.d2, tof=lm.tof, frame=lm.dynamicFrames,
            motion_frame=lm.motionFrames, motion=lm.motionTransforms,
            additive=lm.randoms)

    def c(self) -> L.yrtb_events:
        nm = 0 if self.motion is None else self.motion.numel() // 12
        return L.yrtb_events(_ptr(self.d1), _ptr(self.d2), _ptr(self.lor),
                             _ptr(self.tof), _ptr(self.frame),
                             _ptr(self.motion_frame), _ptr(self.motion), nm,
                             _ptr(self.measurement), _ptr(self.sens),
                             _ptr(self.att), _ptr(self.additive), self.count,
                             _ptr(self.orient))


# ---------------------------------------------------------------- projector --
def release_cached_memory():
    """Return the library's cached device temporaries to the CUDA driver
    (yrtb_release_cached_memory)."""
    L.check(L.lib().yrtb_release_cached_memory())


class DeviceProjector:
    """Owns one yrtb_projector handle (scanner + image grid + options)."""

    def __init__(self, scanner: Scanner, img_params: ImageParams,
                 proj_params: ProjectorParams):
        self.scanner = scanner
        self.img_params = img_params
        self.proj_params = proj_params
        L.lib()
        pp, keep = proj_params._c()
        lut = scanner._custom_lut
        h = ctypes.c_void_p()
        torch.cuda.init()
        L.check(L.lib().yrtb_projector_create(
            ctypes.byref(scanner._c()),
            None if lut is None else lut.ctypes.data,
            ctypes.byref(img_params._c()), ctypes.byref(pp), ctypes.byref(h)))
        self.h = h
        del keep

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                L.lib().yrtb_projector_destroy(h)
            except Exception:
                pass
            self.h = None

    def _check_image(self, img: torch.Tensor, nt=None):
        ip = self.img_params
        if not (img.is_cuda and img.dtype == torch.float32 and img.is_contiguous()):
            raise RuntimeError("images must be contiguous float32 CUDA tensors")
        want = ip.numVoxels * (ip.nt if nt is None else nt)
        if img.numel() != want:
            raise RuntimeError(f"image has {img.numel()} voxels, expected {want}")

    def multiray_offsets(self, count: int) -> torch.Tensor:
        nr = self.proj_params.numRays
        out = torch.zeros((count, 4 * max(nr - 1, 0)), dtype=torch.float32,
                          device="cuda")
        if nr > 1:
            L.check(L.lib().yrtb_multiray_offsets(self.h, count, out.data_ptr(),
                                                  _stream()))
        return out

    def multiray_table(self, count: int):
        """Keep the multi-ray offsets of item indices 0..count-1 in a table
        (yrtb_multiray_table): later projections read them instead of
        re-deriving the generator per event; same values."""
        L.check(L.lib().yrtb_multiray_table(self.h, int(count), _stream()))

    def take_event_errors(self) -> int:
        n = ctypes.c_uint64()
        L.check(L.lib().yrtb_projector_take_event_errors(self.h, ctypes.byref(n)))
        return int(n.value)

    def forward(self, img, ev: DeviceEvents, out=None, rng=None):
        self._check_image(img)
        if out is None:
            out = torch.zeros(ev.count, dtype=torch.float32, device=img.device)
        r = rng or L.yrtb_range(0, 1, 0)
        L.check(L.lib().yrtb_forward(self.h, img.data_ptr(),
                                     ctypes.byref(ev.c()), r, out.data_ptr(),
                                     _stream()))
        return out

    def backward(self, values, ev: DeviceEvents, img=None, rng=None):
        ip = self.img_params
        if img is None:
            img = torch.zeros(ip.shape, dtype=torch.float32, device=values.device)
        self._check_image(img)
        r = rng or L.yrtb_range(0, 1, 0)
        L.check(L.lib().yrtb_backward(self.h, values.data_ptr(),
                                      ctypes.byref(ev.c()), r, img.data_ptr(),
                                      _stream()))
        return img

    def em_step(self, img, em, ev: DeviceEvents, rng=None, global_scale=1.0,
                denom_threshold=1e-35, model=None):
        """Fused EM pass: em += A^T (m / u), u the corrected forward
        projection; with model (a float32 tensor of ev.count), u is also
        written there per event."""
        self._check_image(img)
        self._check_image(em)
        r = rng or L.yrtb_range(0, 1, 0)
        if model is not None:
            L.check(L.lib().yrtb_em_step_model(self.h, img.data_ptr(), em.data_ptr(),
                                               ctypes.byref(ev.c()), r,
                                               float(global_scale),
                                               float(denom_threshold),
                                               model.data_ptr(), _stream()))
            return em
        L.check(L.lib().yrtb_em_step(self.h, img.data_ptr(), em.data_ptr(),
                                     ctypes.byref(ev.c()), r,
                                     float(global_scale),
                                     float(denom_threshold), _stream()))
        return em

    # ------------------------------------------------ launch configuration --
    def set_launch(self, block: int = 256, threads_per_lor: int = 1,
                   bucket_shift: int = 3, order: int = 0, tile_shift: int = 1,
                   vector_groups: int = 2):
        c = L.yrtb_launch_config(int(block), int(threads_per_lor), int(bucket_shift),
                                 int(order), int(tile_shift), int(vector_groups))
        L.check(L.lib().yrtb_projector_set_launch(self.h, ctypes.byref(c)))

    @staticmethod
    def _launch_dict(c) -> dict:
        return {"block": c.block, "threads_per_lor": c.threads_per_lor,
                "bucket_shift": c.bucket_shift, "order": c.order,
                "tile_shift": c.tile_shift, "vector_groups": c.vector_groups}

    def get_launch(self) -> dict:
        c = L.yrtb_launch_config()
        L.check(L.lib().yrtb_projector_get_launch(self.h, ctypes.byref(c)))
        return self._launch_dict(c)

    # --------------------------------------------------------- image layout --
    def set_image_layout(self, layout: int):
        """Layout of the images given to forward / backward / em_step
        (L.YRTB_LAYOUT_ROW_MAJOR or L.YRTB_LAYOUT_TILE_4X2, see
        yrtb_projector_set_image_layout); convert images with to_layout."""
        L.check(L.lib().yrtb_projector_set_image_layout(self.h, int(layout)))

    def get_image_layout(self) -> int:
        v = ctypes.c_int()
        L.check(L.lib().yrtb_projector_get_image_layout(self.h, ctypes.byref(v)))
        return v.value

    @staticmethod
    def to_layout(img: torch.Tensor, img_params: ImageParams, layout: int,
                  out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """img (nt frames, in the other layout) converted to `layout`."""
        src = img.contiguous().reshape(-1)
        if src.numel() != img_params.numVoxels * img_params.nt or \
                src.dtype != torch.float32 or not src.is_cuda:
            raise RuntimeError("image does not match the image parameters")
        if out is None:
            out = torch.empty_like(src)
        L.check(L.lib().yrtb_image_convert_layout(src.data_ptr(), out.data_ptr(),
                                                  ctypes.byref(img_params._c()),
                                                  int(layout), _stream()))
        return out

    def autotune(self, img, ev: DeviceEvents, num_subsets: int = 1,
                 max_sample: int = 2_000_000) -> dict:
        """Time the fused EM step over a sample of the events for every launch
        configuration this projector admits and keep the fastest
        (yrtb_autotune).  Returns {"best": cfg, "sample_events": n,
        "tried": [(cfg, ms), ...]}."""
        self._check_image(img)
        rep = L.yrtb_tune_report()
        L.check(L.lib().yrtb_autotune(self.h, img.data_ptr(), ctypes.byref(ev.c()),
                                      int(num_subsets), int(max_sample),
                                      ctypes.byref(rep), _stream()))
        cfg = self._launch_dict
        return {"best": cfg(rep.best), "sample_events": int(rep.sample_events),
                "tried": [(cfg(rep.tried[i]), float(rep.ms[i]))
                          for i in range(rep.num_tried)]}

    def order_events(self, ev: DeviceEvents, num_subsets: int,
                     first_global_index: int = 0):
        """Subset-major, LOR-sorted copy of the events (yrtb_events_subset_
        order_from + yrtb_events_gather); event e belongs to subset
        (first_global_index + e) mod num_subsets (a shard of a longer stream
        starts at its first event's global index).  Returns (events, subset
        offsets)."""
        n = ev.count
        perm = torch.empty(n, dtype=torch.int64, device="cuda")
        offs = np.zeros(num_subsets + 1, np.uint64)
        L.check(L.lib().yrtb_events_subset_order_from(
            self.h, ctypes.byref(ev.c()), int(num_subsets),
            int(first_global_index), perm.data_ptr(), offs.ctypes.data,
            _stream()))
        like = lambda t: None if t is None else torch.empty_like(t)
        out = DeviceEvents(n, like(ev.d1), like(ev.d2), like(ev.lor),
                           like(ev.tof), like(ev.frame), like(ev.motion_frame),
                           ev.motion, like(ev.measurement), like(ev.sens),
                           like(ev.att), like(ev.additive), orient=like(ev.orient))
        L.check(L.lib().yrtb_events_gather(ctypes.byref(ev.c()), perm.data_ptr(),
                                           ctypes.byref(out.c()), _stream()))
        out.perm = perm
        return out, offs

    def count_crossings(self, ev: DeviceEvents, rng=None) -> torch.Tensor:
        out = torch.zeros(ev.count, dtype=torch.int32, device="cuda")
        r = rng or L.yrtb_range(0, 1, 0)
        L.check(L.lib().yrtb_count_crossings(self.h, ctypes.byref(ev.c()), r,
                                             out.data_ptr(), _stream()))
        return out

    def trace_walks(self, ev: DeviceEvents, cap: int = 1024, rng=None):
        """Visits of each event's forward walk (yrtb_trace_walks): (offsets
        int32 [n, cap], weights float32 [n, cap], counts int32 [n]); row k
        holds the first counts[k] (at most cap) visits of item k in visit
        order."""
        r = rng or L.yrtb_range(0, 1, 0)
        stride = max(1, int(r.stride))
        n = int(r.count) if r.count else max(0, (ev.count - int(r.start) + stride - 1) // stride)
        offs = torch.zeros((n, cap), dtype=torch.int32, device="cuda")
        wts = torch.zeros((n, cap), dtype=torch.float32, device="cuda")
        cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
        L.check(L.lib().yrtb_trace_walks(self.h, ctypes.byref(ev.c()), r, int(cap),
                                         offs.data_ptr(), wts.data_ptr(), cnt.data_ptr(),
                                         _stream()))
        return offs, wts, cnt

    def attenuation_factors(self, mu: torch.Tensor, mu_params: ImageParams,
                            ev: DeviceEvents, out=None, rng=None):
        if out is None:
            out = torch.zeros(ev.count, dtype=torch.float32, device=mu.device)
        r = rng or L.yrtb_range(0, 1, 0)
        L.check(L.lib().yrtb_attenuation_factors(
            self.h, mu.data_ptr(), ctypes.byref(mu_params._c()),
            ctypes.byref(ev.c()), r, out.data_ptr(), _stream()))
        return out

    def gather_histo3d(self, histo: torch.Tensor, ev: DeviceEvents,
                       invert=False, out=None, rng=None):
        if out is None:
            out = torch.zeros(ev.count, dtype=torch.float32, device=histo.device)
        r = rng or L.yrtb_range(0, 1, 0)
        L.check(L.lib().yrtb_gather_histo3d(self.h, histo.data_ptr(),
                                            ctypes.byref(ev.c()), r,
                                            int(bool(invert)), out.data_ptr(),
                                            _stream()))
        return out

    def gather_crystal_product(self, crystal_eff: torch.Tensor,
                               ev: DeviceEvents, out=None, rng=None):
        """Per-event eff[d1] * eff[d2] (LOR sensitivity from crystal factors)."""
        if out is None:
            out = torch.zeros(ev.count, dtype=torch.float32,
                              device=crystal_eff.device)
        r = rng or L.yrtb_range(0, 1, 0)
        L.check(L.lib().yrtb_gather_crystal_product(
            self.h, crystal_eff.data_ptr(), ctypes.byref(ev.c()), r,
            out.data_ptr(), _stream()))
        return out

    def sensitivity_histo3d(self, sens_img, num_subsets=1, subset=0,
                            sens_histo=None, acf_histo=None, mu=None,
                            mu_params: Optional[ImageParams] = None,
                            crystal_eff=None):
        """Back projection of a subset of all histogram bins; the LOR
        sensitivity is sens_histo[bin], or crystal_eff[d1] * crystal_eff[d2]."""
        self._check_image(sens_img, nt=1)
        mp = None if mu_params is None else ctypes.byref(mu_params._c())
        if crystal_eff is not None:
            if sens_histo is not None:
                raise RuntimeError("give a sensitivity histogram or crystal "
                                   "factors, not both")
            L.check(L.lib().yrtb_sensitivity_histo3d_crystal(
                self.h, sens_img.data_ptr(), crystal_eff.data_ptr(),
                _ptr(acf_histo), _ptr(mu), mp, int(num_subsets), int(subset),
                _stream()))
            return sens_img
        L.check(L.lib().yrtb_sensitivity_histo3d(
            self.h, sens_img.data_ptr(), _ptr(sens_histo), _ptr(acf_histo),
            _ptr(mu), mp, int(num_subsets), int(subset), _stream()))
        return sens_img

    def em_step_histo3d(self, img, em, meas, num_subsets, subset,
                        sens_histo=None, acf_histo=None, additive_histo=None,
                        global_scale=1.0, denom_threshold=1e-35, bins=None):
        """Histogram-mode EM pass over one subset; with bins (the list of
        histo3d_subset_nonzero for this subset) only those bins are visited."""
        if bins is not None:
            L.check(L.lib().yrtb_em_step_histo3d_list(
                self.h, img.data_ptr(), em.data_ptr(), meas.data_ptr(),
                _ptr(sens_histo), _ptr(acf_histo), _ptr(additive_histo),
                int(num_subsets), int(subset), bins.data_ptr(), bins.numel(),
                float(global_scale), float(denom_threshold), _stream()))
            return em
        L.check(L.lib().yrtb_em_step_histo3d(
            self.h, img.data_ptr(), em.data_ptr(), meas.data_ptr(),
            _ptr(sens_histo), _ptr(acf_histo), _ptr(additive_histo),
            int(num_subsets), int(subset), float(global_scale),
            float(denom_threshold), _stream()))
        return em

    def histo3d_subset_nonzero(self, meas, num_subsets, subset, capacity):
        """Subset-local indices (int64 tensor, increasing) of the bins of the
        subset with a valid pair and a non-zero measurement; capacity >= the
        subset's bin count."""
        buf = torch.empty(int(capacity), dtype=torch.int64, device=meas.device)
        n = ctypes.c_uint64()
        L.check(L.lib().yrtb_histo3d_subset_nonzero(
            self.h, meas.data_ptr(), int(num_subsets), int(subset), buf.data_ptr(),
            int(capacity), ctypes.byref(n), _stream()))
        return buf[:n.value].clone()


_proj_cache = {}


def histo3d_bins(scanner: Scanner, d1, d2) -> np.ndarray:
    """Histogram3D::getBinIdFromDetPair for arrays (UINT64_MAX = invalid)."""
    p = _scratch_projector(scanner)
    a = _dev(np.atleast_1d(np.asarray(d1, np.uint32)), torch.int32)
    b = _dev(np.atleast_1d(np.asarray(d2, np.uint32)), torch.int32)
    out = torch.empty(a.numel(), dtype=torch.int64, device="cuda")
    L.check(L.lib().yrtb_histo3d_bins(p.h, a.data_ptr(), b.data_ptr(),
                                      a.numel(), out.data_ptr(), _stream()))
    return out.cpu().numpy().view(np.uint64)


def histo3d_detpairs(scanner: Scanner, bins):
    p = _scratch_projector(scanner)
    bb = torch.from_numpy(np.ascontiguousarray(np.atleast_1d(bins),
                                               np.uint64).view(np.int64)).cuda()
    d1 = torch.empty(bb.numel(), dtype=torch.int32, device="cuda")
    d2 = torch.empty_like(d1)
    L.check(L.lib().yrtb_histo3d_detpairs(p.h, bb.data_ptr(), bb.numel(),
                                          d1.data_ptr(), d2.data_ptr(),
                                          _stream()))
    return (d1.cpu().numpy().view(np.uint32), d2.cpu().numpy().view(np.uint32))


def _scratch_projector(scanner: Scanner) -> DeviceProjector:
    key = id(scanner)
    p = _proj_cache.get(key)
    if p is None or p.scanner is not scanner:
        p = DeviceProjector(scanner, ImageParams(1, 1, 1, 1, 1, 1),
                            ProjectorParams(scanner))
        _proj_cache[key] = p
    return p


def convertToHistogram3D(lm: ListModeLUT, values=None) -> Histogram3D:
    """List-mode -> Histogram3D on the GPU (bit-exact float counts)."""
    h = Histogram3D(lm.scanner)
    p = _scratch_projector(lm.scanner)
    ev = lm.device_events()
    histo = torch.zeros(h.histoSize, dtype=torch.float32, device="cuda")
    vals = _dev(values, torch.float32)
    bad = ctypes.c_uint64()
    L.check(L.lib().yrtb_listmode_to_histo3d(
        p.h, ev.d1.data_ptr(), ev.d2.data_ptr(), _ptr(vals), ev.count,
        histo.data_ptr(), ctypes.byref(bad), _stream()))
    h.data = histo.cpu().numpy()
    return h


# --------------------------------------------------- OperatorProjectorDevice --
class ProjectionList:
    """Projection values over the bins of a projection data object, on the
    GPU: the reference's ProjectionListOwned
    (include/yrt-pet/datastruct/projection/ProjectionList.hpp:21-84), one
    float per list-mode event or histogram bin, that
    OperatorProjectorDevice.applyA writes and applyAH reads."""

    def __init__(self, reference):
        self.reference = reference
        self.values: Optional[torch.Tensor] = None

    def allocate(self):
        self.values = torch.zeros(self.reference.count(), dtype=torch.float32,
                                  device="cuda")

    def count(self) -> int:
        return self.reference.count()

    def getBinIter(self, numSubsets: int, idxSubset: int):
        return self.reference.getBinIter(numSubsets, idxSubset)

    def _require(self):
        if self.values is None:
            raise RuntimeError("ProjectionList memory is not allocated")
        return self.values

    def getProjectionValue(self, i: int) -> float:
        return float(self._require()[i])

    def setProjectionValue(self, i: int, v: float):
        self._require()[i] = float(v)

    def clearProjections(self, v: float = 0.0):
        self._require().fill_(float(v))

    def getProjectionsArray(self) -> np.ndarray:
        return self._require().cpu().numpy()


ProjectionListOwned = ProjectionList


class OperatorProjectorDevice:
    """Projection operator A (applyA) and its adjoint (applyAH) over the bins
    of one BinIterator, on the GPU, with the reference's pybind signatures
    (src/operators/OperatorProjectorDevice.cu:26-90): applyA(img, proj)
    writes A img into the ProjectionList proj (its entries outside the bin
    iterator untouched), applyAH(proj, img) adds A^T proj to img.  Images are
    float32 CUDA tensors of the operator's image parameters (create(...,
    img_params=...) or setImageParams)."""

    def __init__(self, proj_params: ProjectorParams, bin_iter=None,
                 img_params: Optional[ImageParams] = None):
        self.proj_params = proj_params
        self.bin_iter = bin_iter
        self.img_params = img_params
        self._proj = None

    @staticmethod
    def create(proj_params: ProjectorParams, bin_iter, constraints=(),
               mem_available: int = 0, img_params: Optional[ImageParams] = None):
        """OperatorProjectorDevice::create (OperatorProjectorDevice.cuh:27-31).
        Detector constraints and a memory budget are not supported: events
        stay resident on the device instead of being loaded in batches, and
        constraints would have to filter them first; both raise."""
        if constraints:
            raise RuntimeError("libyrtb projectors take no detector constraints: "
                               "filter the events before projecting them")
        if mem_available:
            raise RuntimeError("libyrtb projectors keep the events resident on "
                               "the device and take no memory budget "
                               "(mem_available must be 0)")
        return OperatorProjectorDevice(proj_params, bin_iter, img_params)

    def setImageParams(self, img_params: ImageParams):
        self.img_params = img_params

    def getBinIter(self):
        return self.bin_iter

    def setBinIter(self, bin_iter):
        self.bin_iter = bin_iter

    def _projector(self, img_params: Optional[ImageParams] = None) -> DeviceProjector:
        ip = img_params or self.img_params
        if ip is None:
            raise RuntimeError("The operator has no image parameters (give "
                               "img_params to create() or setImageParams)")
        if self._proj is None or self._proj.img_params is not ip:
            self._proj = DeviceProjector(self.proj_params.scanner, ip,
                                         self.proj_params)
        return self._proj

    def _events(self, projData):
        if isinstance(projData, ProjectionList):
            projData = projData.reference
        if isinstance(projData, ListModeLUT):
            return projData.device_events(), self.bin_iter._range()
        if isinstance(projData, Histogram3D):
            bins = self.bin_iter.indices()
            d1, d2 = histo3d_detpairs(projData.scanner, bins)
            ev = DeviceEvents.from_arrays(d1, d2)
            return ev, None
        raise RuntimeError("The Projection Data provided is not a "
                           "ProjectionList, ListModeLUT nor Histogram3D")

    def _check_image(self, img: torch.Tensor, p: DeviceProjector):
        if not isinstance(img, torch.Tensor) or not img.is_cuda:
            raise RuntimeError("The image provided is not a CUDA tensor")
        if img.numel() != p.img_params.nt * p.img_params.numVoxels:
            raise RuntimeError("The image does not match the operator's image "
                               "parameters")

    def applyA(self, img: torch.Tensor, proj: ProjectionList):
        """proj.values[bins of the iterator] = A img."""
        if not isinstance(proj, ProjectionList):
            raise RuntimeError("applyA writes into a ProjectionList "
                               "(ProjectionListOwned(data).allocate())")
        p = self._projector()
        self._check_image(img, p)
        vals = proj._require()
        ev, rng = self._events(proj)
        x = img.contiguous()
        if isinstance(proj.reference, Histogram3D):
            idx = torch.from_numpy(self.bin_iter.indices().astype(np.int64)).to(img.device)
            vals[idx] = p.forward(x, ev)
            return proj
        p.forward(x, ev, out=vals, rng=rng)
        return proj

    def applyAH(self, proj: ProjectionList, img: torch.Tensor):
        """img += A^T proj.values over the bins of the iterator."""
        if not isinstance(proj, ProjectionList):
            raise RuntimeError("applyAH reads a ProjectionList")
        p = self._projector()
        self._check_image(img, p)
        vals = proj._require()
        ev, rng = self._events(proj)
        if isinstance(proj.reference, Histogram3D):
            idx = torch.from_numpy(self.bin_iter.indices().astype(np.int64)).to(vals.device)
            p.backward(vals[idx].contiguous(), ev, img=img)
            return img
        p.backward(vals, ev, img=img, rng=rng)
        return img


class ProjectionOper:
    """numpy A / At wrapper (python/pyyrtpet/_pyyrtpet.py:81-157) on the GPU."""

    def __init__(self, scanner: Scanner, img_params: ImageParams, projData,
                 projector="Siddon", updater_type="DEFAULT4D", idx_subset=0,
                 num_subsets=1, tof_width_ps=None, tof_n_std=0,
                 proj_psf_fname=None, num_rays=1, H_basis=None,
                 update_H=False, use_gpu=True):
        updater_type = getattr(updater_type, "name", str(updater_type)).upper()
        if updater_type not in ("DEFAULT4D", "LR"):
            raise RuntimeError("Projector updater type not valid")
        self._scanner = scanner
        self._img_params = img_params
        self._projData = projData
        self._binIter = projData.getBinIter(num_subsets, idx_subset)
        pp = ProjectorParams(scanner)
        pp.setProjector(projector)
        if tof_width_ps is not None:
            pp.addTOF(tof_width_ps or 0.0, tof_n_std or 0)
        pp.projPsf_fname = proj_psf_fname or ""
        pp.numRays = num_rays
        self._proj_params = pp
        self._oper = OperatorProjectorDevice.create(pp, self._binIter,
                                                    img_params=img_params)
        self._image_shape = img_params.shape
        self._lr = None
        if updater_type == "LR":
            # Low-rank image: x holds rank images W, the frames are
            # x_t = sum_l H[l][t] W_l (the LR updater); events carry their
            # dynamic frame (ListModeLUT.addDynamicFraming).
            if H_basis is None:
                raise RuntimeError("LR updater was requested but HBasis is empty")
            pp.updaterType = "LR"
            pp.setHBasisFromNumpy(H_basis)
            pp.updateH = bool(update_H)
            R, T = pp.HBasis.shape
            self._image_shape = (R,) + img_params.shape[1:]
            self._frames_params = img_params.withFrames(T)

    def _lr_projector(self):
        from .lrem import LowRankProjector
        if self._lr is None:
            dp = self._oper._projector(self._frames_params)
            self._lr = LowRankProjector(dp, self._proj_params.HBasis)
        return self._lr

    def A(self, x):
        xx = torch.as_tensor(np.require(x, np.float32)).reshape(
            self._image_shape).cuda()
        if self._proj_params.updaterType == "LR":
            ev, rng = self._oper._events(self._projData)
            out = torch.zeros(ev.count, dtype=torch.float32, device="cuda")
            return self._lr_projector().forward(xx, ev, out=out, rng=rng).cpu().numpy()
        pl = ProjectionList(self._projData)
        pl.allocate()
        self._oper.applyA(xx, pl)
        return pl.values.cpu().numpy()

    def At(self, y, W=None):
        """Back projection.  With the LR updater: onto W (rank images), or,
        with update_H, onto the temporal basis given the rank images W
        (returns the rank x frames numerator sum value * weight * W[l][j])."""
        yy = torch.as_tensor(np.require(y, np.float32)).cuda()
        if self._proj_params.updaterType == "LR":
            ev, rng = self._oper._events(self._projData)
            lrp = self._lr_projector()
            if self._proj_params.updateH:
                if W is None:
                    raise RuntimeError("the H back projection needs the rank images W")
                Wt = torch.as_tensor(np.require(W, np.float32)).reshape(
                    self._image_shape).cuda()
                return lrp.backward_h(yy, Wt, ev, rng=rng).cpu().numpy()
            return lrp.backward(yy, ev, rng=rng).cpu().numpy()
        pl = ProjectionList(self._projData)
        pl.values = yy.reshape(-1).contiguous()
        x = torch.zeros(self._img_params.shape, dtype=torch.float32, device="cuda")
        self._oper.applyAH(pl, x)
        return x.cpu().numpy()
