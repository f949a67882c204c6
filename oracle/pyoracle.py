"""Test infrastructure: ctypes front-end of the CPU oracle and of the reference.

Two CPU implementations of the YRT-PET projection hot path are reachable from
here, both used only to check results (tests/, ``__graft_entry__.smoke()``)
and to time the CPU baseline (``bench.py``):

* ``liboracle.so``   -- the restatement in ``oracle/oracle.cpp`` (float mirror
  of the reference's FP32 order, and an FP64 oracle);
* ``_ref/libyrtref_harness.so`` -- the YRT-PET 2.0.7 reference library itself,
  compiled from its own sources by ``oracle/ref.mk`` (present only where that
  recipe ran).

and, on a machine with a GPU, the reference's own CUDA path:

* ``_ref_cuda/libyrtref_gpu_harness.so`` -- the same harness built by
  ``oracle/ref_cuda.mk`` against the reference compiled with BUILD_CUDA for
  sm_100a; its OSEM and list-mode projection entry points run OSEM_GPU and
  OperatorProjectorDevice (the functions below take ``gpu=True``).

The product package never imports this module.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libyrtref_harness.so")
REF_GPU_SO = os.path.join(HERE, "_ref_cuda", "libyrtref_gpu_harness.so")
REF_B200_SO = os.path.join(HERE, "_ref_cuda", "libyrtref_b200_harness.so")


class ScannerDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in
                ("axialFOV", "crystalSize_z", "crystalSize_trans",
                 "crystalDepth", "scannerRadius")] + \
               [(n, ctypes.c_uint64) for n in
                ("detsPerRing", "numRings", "numDOI", "maxRingDiff",
                 "minAngDiff", "detsPerBlock")]


class ImageDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("nx", "ny", "nz", "nt")] + \
               [(n, ctypes.c_float) for n in
                ("length_x", "length_y", "length_z", "off_x", "off_y",
                 "off_z")]


class ProjDesc(ctypes.Structure):
    _fields_ = [("projector", ctypes.c_int), ("incremental", ctypes.c_int),
                ("tof_fwhm_ps", ctypes.c_float), ("tof_n_std", ctypes.c_int),
                ("num_rays", ctypes.c_int), ("crystal_z", ctypes.c_float),
                ("crystal_trans", ctypes.c_float),
                ("psf_num_s", ctypes.c_int), ("psf_size", ctypes.c_int),
                ("psf_s_step", ctypes.c_float),
                ("psf_k_spacing", ctypes.c_float),
                ("psf_taps", ctypes.c_void_p), ("threads", ctypes.c_int)]


class LmExtra(ctypes.Structure):
    _fields_ = [("timestamps", ctypes.c_void_p), ("num_frame_ts", ctypes.c_uint64),
                ("frame_ts", ctypes.c_void_p), ("num_motion", ctypes.c_uint64),
                ("motion_starts", ctypes.c_void_p), ("motion", ctypes.c_void_p)]


class OsemDesc(ctypes.Structure):
    _fields_ = [("projector", ctypes.c_int), ("num_rays", ctypes.c_int),
                ("tof_fwhm_ps", ctypes.c_float), ("tof_n_std", ctypes.c_int),
                ("iterations", ctypes.c_int), ("subsets", ctypes.c_int),
                ("threads", ctypes.c_int), ("global_scale", ctypes.c_float),
                ("hard_threshold", ctypes.c_float), ("listmode", ctypes.c_int),
                ("image_psf_csv", ctypes.c_char_p), ("image_psf_variant", ctypes.c_int)]


@dataclass
class Scanner:
    """Arguments of the reference ``Scanner`` constructor (Scanner.cpp:102)."""
    axialFOV: float
    crystalSize_z: float
    crystalSize_trans: float
    crystalDepth: float
    scannerRadius: float
    detsPerRing: int
    numRings: int
    numDOI: int = 1
    maxRingDiff: int = 0
    minAngDiff: int = 1
    detsPerBlock: int = 1

    def desc(self) -> ScannerDesc:
        return ScannerDesc(self.axialFOV, self.crystalSize_z,
                           self.crystalSize_trans, self.crystalDepth,
                           self.scannerRadius, self.detsPerRing, self.numRings,
                           self.numDOI, self.maxRingDiff, self.minAngDiff,
                           self.detsPerBlock)

    @property
    def num_dets(self) -> int:
        return self.detsPerRing * self.numRings * self.numDOI


@dataclass
class ImageParams:
    nx: int
    ny: int
    nz: int
    length_x: float
    length_y: float
    length_z: float
    off_x: float = 0.0
    off_y: float = 0.0
    off_z: float = 0.0
    nt: int = 1

    def desc(self) -> ImageDesc:
        return ImageDesc(self.nx, self.ny, self.nz, self.nt, self.length_x,
                         self.length_y, self.length_z, self.off_x, self.off_y,
                         self.off_z)

    @property
    def shape(self):
        return (self.nt, self.nz, self.ny, self.nx)

    @property
    def num_voxels(self) -> int:
        return self.nx * self.ny * self.nz


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


_oracle = None
_ref = None
_ref_gpu = None
_ref_b200 = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = ctypes.CDLL(ORACLE_SO)
        _oracle.orc_siddon_trace_f32.restype = ctypes.c_int64
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _setup_ref(lib):
    lib.ref_dd_overlap.restype = ctypes.c_float
    lib.ref_dd_overlap.argtypes = [ctypes.c_float] * 4
    lib.ref_last_error.restype = ctypes.c_char_p
    lib.ref_tof.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_float,
                            ctypes.c_float, ctypes.c_float,
                            ctypes.c_float, ctypes.c_void_p]
    return lib


def ref_lib(gpu=False):
    """The reference harness: the CPU build; with gpu=True the build whose
    OSEM and list-mode projections run the reference's CUDA path; with
    gpu="b200" the build whose OSEM and list-mode projections run the
    reference's drivers on the product's binding classes (OSEM_GPU_B200,
    OperatorProjectorB200 over libyrtb)."""
    global _ref, _ref_gpu, _ref_b200
    if gpu == "b200":
        if _ref_b200 is None:
            _ref_b200 = _setup_ref(ctypes.CDLL(REF_B200_SO))
            assert _ref_b200.ref_uses_gpu() == 2
        return _ref_b200
    if gpu:
        if _ref_gpu is None:
            _ref_gpu = _setup_ref(ctypes.CDLL(REF_GPU_SO))
            assert _ref_gpu.ref_uses_gpu() == 1
        return _ref_gpu
    if _ref is None:
        _ref = _setup_ref(ctypes.CDLL(REF_SO))
    return _ref


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


def ref_b200_available() -> bool:
    return os.path.exists(REF_B200_SO)


def ref_set_b200_precision(precision: int):
    """0: mirror, 1: compensated arithmetic for the binding's projections."""
    ref_lib("b200").ref_set_b200_precision(ctypes.c_int(precision))


class _StdoutToStderr:
    """Sends the reference's progress prints (std::cout) to stderr so that
    stdout carries only the caller's own output."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self._saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        import sys
        try:
            ctypes.CDLL(None).fflush(None)
        except Exception:
            pass
        sys.stdout.flush()
        os.dup2(self._saved, 1)
        os.close(self._saved)
        return False


def quiet():
    return _StdoutToStderr()


def _ref_check(rc, gpu=False):
    if rc != 0:
        raise RuntimeError(ref_lib(gpu).ref_last_error().decode())


@dataclass
class Proj:
    """Projector options (reference ProjectorParams subset)."""
    projector: str = "S"          # "S" Siddon, "DD"
    incremental: bool = True
    tof_fwhm_ps: float = 0.0
    tof_n_std: int = 0
    num_rays: int = 1
    crystal_z: float = 0.0
    crystal_trans: float = 0.0
    psf_taps: np.ndarray | None = None   # (num_s, size)
    psf_s_step: float = 0.0
    psf_k_spacing: float = 0.0
    threads: int = 8

    def desc(self) -> ProjDesc:
        taps = self.psf_taps
        if taps is not None:
            taps = np.ascontiguousarray(taps, dtype=np.float32)
            self._taps_keep = taps
        return ProjDesc(0 if self.projector == "S" else 1,
                        int(self.incremental), self.tof_fwhm_ps,
                        self.tof_n_std, self.num_rays, self.crystal_z,
                        self.crystal_trans,
                        0 if taps is None else taps.shape[0],
                        0 if taps is None else taps.shape[1],
                        self.psf_s_step, self.psf_k_spacing,
                        None if taps is None else taps.ctypes.data,
                        self.threads)


# ------------------------------------------------------------ oracle calls --
def scanner_lut(sc: Scanner) -> np.ndarray:
    out = np.zeros((sc.num_dets, 6), np.float32)
    oracle_lib().orc_scanner_lut(ctypes.byref(sc.desc()), _p(out))
    return out


def histo3d_dims(sc: Scanner):
    dims = np.zeros(3, np.uint64)
    oracle_lib().orc_histo3d_dims(ctypes.byref(sc.desc()), _p(dims))
    return tuple(int(x) for x in dims)


def histo3d_bins(sc: Scanner, d1, d2) -> np.ndarray:
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    out = np.zeros(len(d1), np.uint64)
    oracle_lib().orc_histo3d_bins(ctypes.byref(sc.desc()),
                                  ctypes.c_uint64(len(d1)), _p(d1), _p(d2),
                                  _p(out))
    return out


def histo3d_detpairs(sc: Scanner, bins):
    bins = _c(bins, np.uint64)
    d1 = np.zeros(len(bins), np.uint32)
    d2 = np.zeros(len(bins), np.uint32)
    oracle_lib().orc_histo3d_detpairs(ctypes.byref(sc.desc()),
                                      ctypes.c_uint64(len(bins)), _p(bins),
                                      _p(d1), _p(d2))
    return d1, d2


def lm_to_histo3d(sc: Scanner, d1, d2, values=None):
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    values = _c(values, np.float32)
    histo = np.zeros(int(np.prod(histo3d_dims(sc))), np.float32)
    bad = ctypes.c_uint64()
    oracle_lib().orc_lm_to_histo3d(ctypes.byref(sc.desc()),
                                   ctypes.c_uint64(len(d1)), _p(d1), _p(d2),
                                   _p(values), _p(histo), ctypes.byref(bad))
    return histo, int(bad.value)


def tof_f32(fwhm, nstd, lor_norm, tof, lo, hi):
    out = np.zeros(6, np.float32)
    f = ctypes.c_float
    oracle_lib().orc_tof_f32(f(fwhm), ctypes.c_int(nstd), f(lor_norm), f(tof),
                             f(lo), f(hi), _p(out))
    return out


def project(ip: ImageParams, pr: Proj, lors, *, image=None, values=None,
            orients=None, tof=None, frames=None, ray_offsets=None,
            forward=True, precision="f32"):
    """Oracle projection. forward: returns values; else returns the image."""
    lib = oracle_lib()
    lors = _c(lors, np.float32)
    n = len(lors)
    orients = _c(orients, np.float32)
    tof = _c(tof, np.float32)
    frames = _c(frames, np.int32)
    ray_offsets = _c(ray_offsets, np.float32)
    dt = np.float32 if precision == "f32" else np.float64
    fn = lib.orc_project_f32 if precision == "f32" else lib.orc_project_f64
    pd = pr.desc()
    if forward:
        img = _c(image, np.float32)
        out = np.zeros(n, dt)
        fn(ctypes.byref(ip.desc()), ctypes.byref(pd), ctypes.c_uint64(n),
           _p(lors), _p(orients), _p(tof), _p(frames), _p(ray_offsets),
           _p(img), 1, _p(out), None)
        return out
    vals = _c(values, dt)
    out = np.zeros(ip.shape, dt)
    fn(ctypes.byref(ip.desc()), ctypes.byref(pd), ctypes.c_uint64(n),
       _p(lors), _p(orients), _p(tof), _p(frames), _p(ray_offsets), None, 0,
       _p(vals), _p(out))
    return out


def siddon_trace(ip: ImageParams, pr: Proj, lor, tof=0.0, cap=1 << 16):
    lor = _c(lor, np.float32)
    idx = np.zeros(cap, np.int64)
    w = np.zeros(cap, np.float32)
    k = oracle_lib().orc_siddon_trace_f32(
        ctypes.byref(ip.desc()), ctypes.byref(pr.desc()), _p(lor),
        ctypes.c_float(tof), _p(idx), _p(w), ctypes.c_int64(cap))
    return idx[:k], w[:k]


def siddon_trace_f64(ip: ImageParams, pr: Proj, lor, tof=0.0, cap=1 << 16):
    lib = oracle_lib()
    lib.orc_siddon_trace_f64.restype = ctypes.c_int64
    lor = _c(lor, np.float32)
    idx = np.zeros(cap, np.int64)
    w = np.zeros(cap, np.float64)
    k = lib.orc_siddon_trace_f64(
        ctypes.byref(ip.desc()), ctypes.byref(pr.desc()), _p(lor),
        ctypes.c_float(tof), _p(idx), _p(w), ctypes.c_int64(cap))
    return idx[:k], w[:k]


def em_step_f64(ip: ImageParams, pr: Proj, lors, image, *, orients=None,
                tof=None, frames=None, ray_offsets=None, measurement=None,
                sens=None, att=None, additive=None, global_scale=1.0,
                denom_thr=1e-35):
    lib = oracle_lib()
    lors = _c(lors, np.float32)
    args = [_c(a, np.float32) for a in
            (orients, tof)] + [_c(frames, np.int32), _c(ray_offsets,
                                                          np.float32)]
    extra = [_c(a, np.float32) for a in (measurement, sens, att, additive)]
    img = _c(image, np.float32)
    out = np.zeros(ip.shape, np.float64)
    lib.orc_em_step_f64(ctypes.byref(ip.desc()), ctypes.byref(pr.desc()),
                        ctypes.c_uint64(len(lors)), _p(lors),
                        *[_p(a) for a in args], *[_p(a) for a in extra],
                        ctypes.c_float(global_scale), ctypes.c_float(denom_thr),
                        _p(img), _p(out))
    return out


def lors_from_detpairs(lut: np.ndarray, d1, d2):
    """LOR endpoints (ProjectionData::getLOR without motion) and orientations."""
    d1 = np.asarray(d1, np.int64)
    d2 = np.asarray(d2, np.int64)
    lors = np.concatenate([lut[d1, :3], lut[d2, :3]], axis=1)
    ori = np.concatenate([lut[d1, 3:], lut[d2, 3:]], axis=1)
    return np.ascontiguousarray(lors), np.ascontiguousarray(ori)


# --------------------------------------------------------- reference calls --
def ref_scanner_lut(sc: Scanner) -> np.ndarray:
    out = np.zeros((sc.num_dets, 6), np.float32)
    _ref_check(ref_lib().ref_scanner_lut(ctypes.byref(sc.desc()), _p(out)))
    return out


def ref_histo3d_dims(sc: Scanner):
    dims = np.zeros(3, np.uint64)
    _ref_check(ref_lib().ref_histo3d_dims(ctypes.byref(sc.desc()), _p(dims)))
    return tuple(int(x) for x in dims)


def ref_histo3d_bins(sc: Scanner, d1, d2):
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    out = np.zeros(len(d1), np.uint64)
    _ref_check(ref_lib().ref_histo3d_bins(ctypes.byref(sc.desc()),
                                          ctypes.c_uint64(len(d1)), _p(d1),
                                          _p(d2), _p(out)))
    return out


def ref_histo3d_detpairs(sc: Scanner, bins):
    bins = _c(bins, np.uint64)
    d1 = np.zeros(len(bins), np.uint32)
    d2 = np.zeros(len(bins), np.uint32)
    _ref_check(ref_lib().ref_histo3d_detpairs(ctypes.byref(sc.desc()),
                                              ctypes.c_uint64(len(bins)),
                                              _p(bins), _p(d1), _p(d2)))
    return d1, d2


def ref_histo3d_crystal_product(sc: Scanner, eff, threads=8, gpu=False):
    """Sensitivity histogram eff[d1] * eff[d2] over every bin, through the
    reference's Histogram3D bin -> detector-pair map."""
    nz, nphi, nr = ref_histo3d_dims(sc)
    out = np.empty(int(nz) * int(nphi) * int(nr), np.float32)
    e = _c(eff, np.float32)
    _ref_check(ref_lib(gpu).ref_histo3d_crystal_product(
        ctypes.byref(sc.desc()), _p(e), ctypes.c_int(threads), _p(out)), gpu)
    return out


def ref_tof(fwhm, nstd, lor_norm, tof, lo, hi):
    out = np.zeros(6, np.float32)
    ref_lib().ref_tof(fwhm, nstd, lor_norm, tof, lo, hi, _p(out))
    return out


def ref_siddon(sc: Scanner, ip: ImageParams, lors, *, image=None, values=None,
               orients=None, tof=None, tof_fwhm_ps=0.0, tof_n_std=0,
               frames=None, num_rays=1, forward=True, incremental=True,
               threads=8):
    lors = _c(lors, np.float32)
    n = len(lors)
    orients = _c(orients, np.float32)
    tof = _c(tof, np.float32)
    frames = _c(frames, np.int32)
    if forward:
        img = np.ascontiguousarray(image, np.float32).copy()
        vals = np.zeros(n, np.float32)
    else:
        img = np.zeros(ip.shape, np.float32)
        vals = np.ascontiguousarray(values, np.float32).copy()
    with quiet():
        rc = ref_lib().ref_siddon(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), _p(img),
            ctypes.c_uint64(n), _p(lors), _p(orients), _p(tof),
            ctypes.c_float(tof_fwhm_ps), ctypes.c_int(tof_n_std), _p(frames),
            ctypes.c_int(num_rays), ctypes.c_int(int(forward)),
            ctypes.c_int(int(incremental)), ctypes.c_int(threads), _p(vals))
    _ref_check(rc)
    return vals if forward else img


def ref_dd(sc: Scanner, ip: ImageParams, lors, orients, *, image=None,
           values=None, tof=None, tof_fwhm_ps=0.0, tof_n_std=0, psf_csv=None,
           forward=True, threads=8):
    lors = _c(lors, np.float32)
    n = len(lors)
    orients = _c(orients, np.float32)
    tof = _c(tof, np.float32)
    if forward:
        img = np.ascontiguousarray(image, np.float32).copy()
        vals = np.zeros(n, np.float32)
    else:
        img = np.zeros(ip.shape, np.float32)
        vals = np.ascontiguousarray(values, np.float32).copy()
    psf = None if psf_csv is None else psf_csv.encode()
    with quiet():
        rc = ref_lib().ref_dd(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), _p(img),
            ctypes.c_uint64(n), _p(lors), _p(orients), _p(tof),
            ctypes.c_float(tof_fwhm_ps), ctypes.c_int(tof_n_std), psf,
            ctypes.c_int(int(forward)), ctypes.c_int(threads), _p(vals))
    _ref_check(rc)
    return vals if forward else img


def ref_read_listmode(sc: Scanner, fname: str, tof: bool, randoms: bool,
                      cap: int):
    L = ref_lib()
    L.ref_read_listmode.restype = ctypes.c_int64
    ts = np.zeros(cap, np.uint32)
    d1 = np.zeros(cap, np.uint32)
    d2 = np.zeros(cap, np.uint32)
    tv = np.zeros(cap, np.float32)
    rv = np.zeros(cap, np.float32)
    with quiet():
        n = L.ref_read_listmode(ctypes.byref(sc.desc()), fname.encode(),
                                int(tof), int(randoms), ctypes.c_uint64(cap),
                                _p(ts), _p(d1), _p(d2), _p(tv), _p(rv))
    if n < 0:
        raise RuntimeError(ref_lib().ref_last_error().decode())
    n = min(n, cap)
    return ts[:n], d1[:n], d2[:n], tv[:n], rv[:n]


def ref_dd_overlap(p0, p1, d0, d1) -> float:
    return ref_lib().ref_dd_overlap(p0, p1, d0, d1)


def ref_lm_to_histo3d(sc: Scanner, d1, d2, threads=8):
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    histo = np.zeros(int(np.prod(ref_histo3d_dims(sc))), np.float32)
    sec = ctypes.c_double()
    with quiet():
        rc = ref_lib().ref_lm_to_histo3d(
            ctypes.byref(sc.desc()), ctypes.c_uint64(len(d1)), _p(d1), _p(d2),
            ctypes.c_int(threads), _p(histo), ctypes.byref(sec))
    _ref_check(rc)
    return histo, sec.value


def _osem_desc(projector="S", num_rays=1, tof_fwhm_ps=0.0, tof_n_std=0,
               iterations=1, subsets=1, threads=8, global_scale=1.0,
               hard_threshold=1.0, listmode=True, image_psf_csv=None,
               image_psf_variant=False):
    return OsemDesc(0 if projector == "S" else 1, num_rays, tof_fwhm_ps,
                    tof_n_std, iterations, subsets, threads, global_scale,
                    hard_threshold, int(listmode),
                    None if image_psf_csv is None else image_psf_csv.encode(),
                    int(bool(image_psf_variant)))


def ref_sensitivity(sc: Scanner, ip: ImageParams, *, sens_histo=None,
                    att_params: ImageParams | None = None, att_image=None,
                    psf_csv=None, gpu=False, **kw):
    o = _osem_desc(**kw)
    nsub = 1 if o.listmode else o.subsets
    out = np.zeros((nsub, ip.nz, ip.ny, ip.nx), np.float32)
    sec = ctypes.c_double()
    sh = _c(sens_histo, np.float32)
    att = _c(att_image, np.float32)
    with quiet():
        rc = ref_lib(gpu).ref_sensitivity(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), ctypes.byref(o),
            _p(sh), None if att_params is None else ctypes.byref(att_params.desc()),
            _p(att), None if psf_csv is None else psf_csv.encode(), _p(out),
            ctypes.byref(sec))
    _ref_check(rc, gpu)
    return out, sec.value


def ref_osem_listmode(sc: Scanner, ip: ImageParams, sens, d1, d2, *, tof=None,
                      randoms=None, sens_histo=None,
                      att_params: ImageParams | None = None, att_image=None,
                      gpu=False, **kw):
    o = _osem_desc(**kw)
    out = np.zeros(ip.shape, np.float32)
    sec = ctypes.c_double()
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    tof = _c(tof, np.float32)
    randoms = _c(randoms, np.float32)
    sh = _c(sens_histo, np.float32)
    att = _c(att_image, np.float32)
    s = _c(sens, np.float32)
    with quiet():
        rc = ref_lib(gpu).ref_osem_listmode(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), ctypes.byref(o),
            _p(s), ctypes.c_uint64(len(d1)), _p(d1), _p(d2), _p(tof), _p(randoms),
            _p(sh), None if att_params is None else ctypes.byref(att_params.desc()),
            _p(att), _p(out), ctypes.byref(sec))
    _ref_check(rc, gpu)
    return out, sec.value


def ref_osem_listmode_dynamic(sc: Scanner, ip: ImageParams, sens, d1, d2,
                              timestamps, *, frame_ts=None, motion_starts=None,
                              motion=None, tof=None, gpu=False, **kw):
    """Reference OSEM with DynamicFraming and/or LORMotion; ip.nt must equal
    the number of dynamic frames (len(frame_ts) - 1)."""
    o = _osem_desc(**kw)
    out = np.zeros(ip.shape, np.float32)
    sec = ctypes.c_double()
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    ts = _c(timestamps, np.uint32)
    fts = _c(frame_ts, np.uint32)
    ms = _c(motion_starts, np.uint32)
    mo = _c(motion, np.float32)
    tof = _c(tof, np.float32)
    s = _c(sens, np.float32)
    ex = LmExtra(ts.ctypes.data, 0 if fts is None else len(fts),
                 None if fts is None else fts.ctypes.data,
                 0 if ms is None else len(ms),
                 None if ms is None else ms.ctypes.data,
                 None if mo is None else mo.ctypes.data)
    with quiet():
        rc = ref_lib(gpu).ref_osem_listmode_ex(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), ctypes.byref(o),
            _p(s), ctypes.c_uint64(len(d1)), _p(d1), _p(d2), _p(tof), None,
            None, None, None, ctypes.byref(ex), _p(out), ctypes.byref(sec))
    _ref_check(rc, gpu)
    return out, sec.value


def ref_osem_histo3d(sc: Scanner, ip: ImageParams, sens_images, histo, *,
                     psf_csv=None, gpu=False, **kw):
    o = _osem_desc(listmode=False, **kw)
    out = np.zeros((ip.nz, ip.ny, ip.nx), np.float32)
    sec = ctypes.c_double()
    s = _c(sens_images, np.float32)
    h = _c(histo, np.float32)
    with quiet():
        rc = ref_lib(gpu).ref_osem_histo3d(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), ctypes.byref(o),
            _p(s), _p(h), None if psf_csv is None else psf_csv.encode(), _p(out),
            ctypes.byref(sec))
    _ref_check(rc, gpu)
    return out, sec.value


def ref_project_lm(sc: Scanner, ip: ImageParams, d1, d2, *, tof=None,
                   image=None, values=None, fwd=True, psf_csv=None,
                   gpu=False, **kw):
    """List-mode forward (values = A x) or back projection (image + A^T v)
    through the reference's util::forwProject / util::backProject, on its CPU
    projector or, with gpu=True, on OperatorProjectorDevice (its CUDA
    kernels).  kw: projector ("S" / "DD"), num_rays, tof_fwhm_ps, tof_n_std,
    threads."""
    o = _osem_desc(**kw)
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    n = len(d1)
    tof = _c(tof, np.float32)
    img = (np.zeros(ip.shape, np.float32) if image is None
           else np.ascontiguousarray(image, np.float32).copy())
    vals = (np.zeros(n, np.float32) if values is None
            else np.ascontiguousarray(values, np.float32).copy())
    with quiet():
        rc = ref_lib(gpu).ref_project_lm(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), _p(img),
            ctypes.c_uint64(n), _p(d1), _p(d2), _p(tof), ctypes.byref(o),
            None if psf_csv is None else psf_csv.encode(), ctypes.c_int(int(fwd)),
            _p(vals))
    _ref_check(rc, gpu)
    return vals if fwd else img


# ------------------------------------------------------ image-space PSF ---
def psf_convolve(ip: ImageParams, image, kx, ky, kz, adjoint=False,
                 precision="f32"):
    """Oracle separable PSF convolution (OperatorPsf::convolve restated)."""
    img = np.ascontiguousarray(image, np.float32)
    kx, ky, kz = (np.ascontiguousarray(k, np.float32) for k in (kx, ky, kz))
    dt = np.float32 if precision == "f32" else np.float64
    out = np.zeros(img.shape, dt)
    fn = (oracle_lib().orc_psf_convolve_f32 if precision == "f32"
          else oracle_lib().orc_psf_convolve_f64)
    rc = fn(ctypes.c_int64(ip.nx), ctypes.c_int64(ip.ny), ctypes.c_int64(ip.nz),
            ctypes.c_int64(ip.nt), _p(img), _p(out), _p(kx), ctypes.c_int(len(kx)),
            _p(ky), ctypes.c_int(len(ky)), _p(kz), ctypes.c_int(len(kz)),
            ctypes.c_int(int(adjoint)))
    assert rc == 0
    return out


def ref_psf_convolve(ip: ImageParams, image, kx, ky, kz, adjoint=False):
    """The reference's OperatorPsf::applyA / applyAH."""
    img = np.ascontiguousarray(image, np.float32)
    kx, ky, kz = (np.ascontiguousarray(k, np.float32) for k in (kx, ky, kz))
    out = np.zeros(img.shape, np.float32)
    with quiet():
        rc = ref_lib().ref_psf_convolve(
            ctypes.byref(ip.desc()), _p(img), _p(out), _p(kx), ctypes.c_int(len(kx)),
            _p(ky), ctypes.c_int(len(ky)), _p(kz), ctypes.c_int(len(kz)),
            ctypes.c_int(int(adjoint)))
    _ref_check(rc)
    return out


def ref_psf_gaussian_kernel(sigma, voxel, size=0):
    """The reference's OperatorPsf::createGaussianKernel1D."""
    buf = np.zeros(4096, np.float32)
    n = ctypes.c_uint64()
    with quiet():
        rc = ref_lib().ref_psf_gaussian_kernel(
            ctypes.c_float(sigma), ctypes.c_float(voxel), ctypes.c_uint64(size),
            _p(buf), ctypes.c_uint64(len(buf)), ctypes.byref(n))
    _ref_check(rc)
    return buf[:n.value].copy()


# ------------------------------------------------------ low-rank images ----
def lr_expand(W, H):
    """Frames of a low-rank image, x_t = sum_l W_l H[l][t] with FP32 products
    and sums in l order (ProjectorUpdaterLR::forwardUpdate,
    src/operators/ProjectorUpdater.cpp:228-243).  W: (R, ...) float32,
    H: (R, T).  Returns (T, ...)."""
    W = np.ascontiguousarray(W, np.float32)
    H = np.ascontiguousarray(H, np.float32)
    R, T = H.shape
    out = np.zeros((T,) + W.shape[1:], np.float32)
    for t in range(T):
        acc = np.zeros(W.shape[1:], np.float32)
        for l in range(R):
            acc = (acc + (W[l] * H[l, t]).astype(np.float32)).astype(np.float32)
        out[t] = acc
    return out


def lr_contract_w_f64(E, H):
    """W-side back projection of a low-rank image from a frame-indexed one:
    Wn_l = sum_t H[l][t] E_t, in FP64 (the reference adds H[l][t] times each
    crossing's value, ProjectorUpdater.cpp:245-266)."""
    E = np.asarray(E, np.float64)
    H = np.asarray(H, np.float64)
    return np.tensordot(H, E, (1, 0))


def lr_contract_h_f64(W, E):
    """H-side back projection: Hn[l][t] = sum_j W[l][j] E[t][j], in FP64."""
    W = np.asarray(W, np.float64).reshape(W.shape[0], -1)
    E = np.asarray(E, np.float64).reshape(E.shape[0], -1)
    return W @ E.T


def ref_siddon_lr(sc: Scanner, ip: ImageParams, lors, frames, H, *, image=None,
                  values=None, tof=None, tof_fwhm_ps=0.0, tof_n_std=0,
                  forward=True, threads=8):
    """The reference's incremental Siddon with its LR updater: ip.nt = rank
    (image = W), H: rank x frames, frames[i] = each LOR's dynamic frame."""
    lors = _c(lors, np.float32)
    n = len(lors)
    tof = _c(tof, np.float32)
    frames = _c(frames, np.int32)
    Hc = np.ascontiguousarray(H, np.float32).copy()
    R, T = Hc.shape
    if forward:
        img = np.ascontiguousarray(image, np.float32).copy()
        vals = np.zeros(n, np.float32)
    else:
        img = np.zeros(ip.shape, np.float32)
        vals = np.ascontiguousarray(values, np.float32).copy()
    with quiet():
        rc = ref_lib().ref_siddon_lr(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), _p(img),
            ctypes.c_uint64(n), _p(lors), _p(tof), ctypes.c_float(tof_fwhm_ps),
            ctypes.c_int(tof_n_std), _p(frames), _p(Hc), ctypes.c_int(R),
            ctypes.c_int(T), ctypes.c_int(int(forward)), ctypes.c_int(threads),
            _p(vals))
    _ref_check(rc)
    return vals if forward else img


def ref_lrem_listmode(sc: Scanner, ip: ImageParams, sens, d1, d2, timestamps,
                      frame_ts, H, *, tof=None, update_h=False, init=None, **kw):
    """Reference low-rank EM (LREM_CPU): ip.nt = rank.  Returns (W, H after
    the reconstruction, seconds); H changes only with update_h."""
    o = _osem_desc(**kw)
    out = np.zeros(ip.shape, np.float32)
    sec = ctypes.c_double()
    d1 = _c(d1, np.uint32)
    d2 = _c(d2, np.uint32)
    ts = _c(timestamps, np.uint32)
    fts = _c(frame_ts, np.uint32)
    tof = _c(tof, np.float32)
    s = _c(sens, np.float32)
    Hc = np.ascontiguousarray(H, np.float32).copy()
    R, T = Hc.shape
    ini = _c(init, np.float32)
    with quiet():
        rc = ref_lib().ref_lrem_listmode(
            ctypes.byref(sc.desc()), ctypes.byref(ip.desc()), ctypes.byref(o),
            _p(s), ctypes.c_uint64(len(d1)), _p(d1), _p(d2), _p(tof), _p(ts),
            _p(fts), _p(Hc), ctypes.c_int(R), ctypes.c_int(T),
            ctypes.c_int(int(update_h)), _p(ini), _p(out), ctypes.byref(sec))
    _ref_check(rc)
    return out, Hc, sec.value


# -------------------------------------------- spatially variant image PSF --
def ref_varpsf_gaussian_kernel(sigmas, nstd, ip: ImageParams):
    """The reference's ConvolutionKernelGaussian (3 sigmas) or
    ConvolutionKernelGaussianMixture (7 values): (weights (z, y, x), half
    sizes (x, y, z))."""
    sig = np.ascontiguousarray(sigmas, np.float32)
    ns = np.ascontiguousarray(nstd, np.float32)
    half = np.zeros(3, np.int32)
    size = ctypes.c_uint64()
    cap = 1 << 20
    out = np.zeros(cap, np.float32)
    rc = ref_lib().ref_varpsf_gaussian_kernel(
        _p(sig), ctypes.c_int(len(sig)), _p(ns), ctypes.byref(ip.desc()), _p(out),
        ctypes.c_uint64(cap), _p(half), ctypes.byref(size))
    _ref_check(rc)
    hx, hy, hz = (int(v) for v in half)
    return out[:size.value].reshape(2 * hz + 1, 2 * hy + 1, 2 * hx + 1).copy(), (hx, hy, hz)


def ref_varpsf_apply(ip: ImageParams, csv: str, image, adjoint=False, threads=8):
    """OperatorVarPsf(csv, params).applyA / applyAH (output zeroed first)."""
    img = np.ascontiguousarray(image, np.float32)
    out = np.zeros(img.shape, np.float32)
    with quiet():
        rc = ref_lib().ref_varpsf_apply(ctypes.byref(ip.desc()), csv.encode(), _p(img),
                                        _p(out), ctypes.c_int(int(adjoint)),
                                        ctypes.c_int(threads))
    _ref_check(rc)
    return out


def varpsf_apply_f64(ip: ImageParams, image, kernels, half_sizes, rng_gap, adjoint=False):
    """FP64 restatement of OperatorVarPsf::varconvolve (one frame): kernels[i]
    (z, y, x) with half sizes (x, y, z); rng_gap = (range x y z, gap x y z).
    Pure-Python loops over the voxels: small images only."""
    img = np.asarray(image, np.float64).reshape(ip.nz, ip.ny, ip.nx)
    nx, ny, nz = ip.nx, ip.ny, ip.nz
    f32 = np.float32
    vx = f32(f32(ip.length_x) / f32(nx))
    vy = f32(f32(ip.length_y) / f32(ny))
    vz = f32(f32(ip.length_z) / f32(nz))
    cx, cy, cz = (f32(f32(n) * v / f32(2)) for n, v in ((nx, vx), (ny, vy), (nz, vz)))
    rx, ry, rz, gx, gy, gz = (f32(v) for v in rng_gap)
    dims = [int(np.floor(f32(r / g))) + 1 for r, g in ((rx, gx), (ry, gy), (rz, gz))]

    def lut(i, j, k):
        t = [f32(abs((i + 0.5) * float(vx) - float(cx))),
             f32(abs((j + 0.5) * float(vy) - float(cy))),
             f32(abs((k + 0.5) * float(vz) - float(cz)))]
        idx = []
        for a, (tv, g) in enumerate(zip(t, (gx, gy, gz))):
            q = f32(tv / g)
            r = int(np.floor(float(q) + 0.5))  # round half away from zero (q >= 0)
            idx.append(min(r, dims[a] - 1))
        return idx[0] + dims[0] * (idx[1] + dims[1] * idx[2])

    out = np.zeros_like(img)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                ki = lut(i, j, k)
                w = np.asarray(kernels[ki], np.float64)
                hx, hy, hz = half_sizes[ki]
                zz = (k + np.arange(-hz, hz + 1)) % nz
                yy = (j + np.arange(-hy, hy + 1)) % ny
                xx = (i + np.arange(-hx, hx + 1)) % nx
                if not adjoint:
                    out[k, j, i] = np.sum(img[np.ix_(zz, yy, xx)] * w)
                else:
                    out[np.ix_(zz, yy, xx)] += img[k, j, i] * w
    return out
