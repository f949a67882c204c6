"""ctypes binding of libyrtb.so (the C ABI declared in include/yrt_b200.h).

The library is loaded from yrt-pet_b200/lib/.  There is no fallback: if the
CUDA library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libyrtb.so")

YRTB_OK = 0
YRTB_ERR_ARGUMENT = 1
YRTB_ERR_CUDA = 2
YRTB_ERR_RANGE = 3
YRTB_ERR_EVENT = 4

YRTB_SIDDON = 0
YRTB_DD = 1
YRTB_OSEM_STATIC_MAX_FLOATS = 4 * 1024 * 1024
YRTB_MIRROR = 0
YRTB_COMPENSATED = 1
YRTB_ORDER_LOR = 0
YRTB_LAYOUT_ROW_MAJOR = 0
YRTB_LAYOUT_TILE_4X2 = 1
YRTB_ORDER_SPATIAL = 1
YRTB_ORDER_SPATIAL_FINE = 2

c_f = ctypes.c_float
c_u64 = ctypes.c_uint64
c_i64 = ctypes.c_int64
c_vp = ctypes.c_void_p


class yrtb_scanner(ctypes.Structure):
    _fields_ = [("axial_fov", c_f), ("crystal_size_z", c_f),
                ("crystal_size_trans", c_f), ("crystal_depth", c_f),
                ("scanner_radius", c_f), ("dets_per_ring", c_u64),
                ("num_rings", c_u64), ("num_doi", c_u64),
                ("max_ring_diff", c_u64), ("min_ang_diff", c_u64),
                ("dets_per_block", c_u64)]


class yrtb_image_params(ctypes.Structure):
    _fields_ = [("nx", c_i64), ("ny", c_i64), ("nz", c_i64), ("nt", c_i64),
                ("length_x", c_f), ("length_y", c_f), ("length_z", c_f),
                ("off_x", c_f), ("off_y", c_f), ("off_z", c_f)]


class yrtb_projector_params(ctypes.Structure):
    _fields_ = [("projector", ctypes.c_int), ("num_rays", ctypes.c_int),
                ("tof_fwhm_ps", c_f), ("tof_n_std", ctypes.c_int),
                ("psf_num_s", ctypes.c_int), ("psf_size", ctypes.c_int),
                ("psf_s_step", c_f), ("psf_k_spacing", c_f),
                ("psf_taps", c_vp), ("precision", ctypes.c_int),
                ("deterministic", ctypes.c_int)]


class yrtb_events(ctypes.Structure):
    _fields_ = [("d1", c_vp), ("d2", c_vp), ("lor", c_vp), ("tof_ps", c_vp),
                ("frame", c_vp), ("motion_frame", c_vp), ("motion", c_vp),
                ("num_motion_frames", c_u64), ("measurement", c_vp), ("sens", c_vp), ("att", c_vp),
                ("additive", c_vp), ("count", c_u64), ("orient", c_vp)]


class yrtb_row_layout(ctypes.Structure):
    _fields_ = [("row_bytes", ctypes.c_uint32)] + \
               [(n, ctypes.c_int32) for n in
                ("lor", "det_orient", "tof", "dynamic_frame", "measurement",
                 "sensitivity", "attenuation", "randoms", "scatter")]


class yrtb_range(ctypes.Structure):
    _fields_ = [("start", c_u64), ("stride", c_u64), ("count", c_u64)]


class yrtb_osem_params(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("subsets", ctypes.c_int),
                ("global_scale", c_f), ("denom_threshold", c_f),
                ("em_threshold", c_f), ("init_from_image", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("d_frame_scale", c_vp),
                ("subset_offsets", c_vp), ("psf", c_vp), ("varpsf", c_vp)]


class yrtb_launch_config(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("threads_per_lor", ctypes.c_int),
                ("bucket_shift", ctypes.c_int), ("order", ctypes.c_int),
                ("tile_shift", ctypes.c_int), ("vector_groups", ctypes.c_int)]


YRTB_TUNE_MAX = 64


class yrtb_tune_report(ctypes.Structure):
    _fields_ = [("best", yrtb_launch_config), ("num_tried", ctypes.c_int),
                ("sample_events", c_u64),
                ("tried", yrtb_launch_config * YRTB_TUNE_MAX),
                ("ms", c_f * YRTB_TUNE_MAX)]


# (name, argtypes) of every entry point of include/yrt_b200.h.
_P = ctypes.POINTER
SIGNATURES = {
    "yrtb_last_error": ([], ctypes.c_char_p),
    "yrtb_version": ([], ctypes.c_int),
    "yrtb_projector_take_event_errors": ([c_vp, _P(c_u64)], ctypes.c_int),
    "yrtb_scanner_regular_lut": ([_P(yrtb_scanner), c_vp], ctypes.c_int),
    "yrtb_histo3d_dims": ([_P(yrtb_scanner), c_vp], ctypes.c_int),
    "yrtb_projector_create": ([_P(yrtb_scanner), c_vp, _P(yrtb_image_params),
                               _P(yrtb_projector_params), _P(c_vp)],
                              ctypes.c_int),
    "yrtb_projector_destroy": ([c_vp], None),
    "yrtb_projector_set_launch": ([c_vp, _P(yrtb_launch_config)], ctypes.c_int),
    "yrtb_projector_get_launch": ([c_vp, _P(yrtb_launch_config)], ctypes.c_int),
    "yrtb_projector_set_image_layout": ([c_vp, ctypes.c_int], ctypes.c_int),
    "yrtb_trace_walks": ([c_vp, _P(yrtb_events), yrtb_range, ctypes.c_uint32, c_vp, c_vp,
                          c_vp, c_vp], ctypes.c_int),
    "yrtb_projector_get_image_layout": ([c_vp, _P(ctypes.c_int)], ctypes.c_int),
    "yrtb_image_convert_layout": ([c_vp, c_vp, _P(yrtb_image_params), ctypes.c_int, c_vp],
                                  ctypes.c_int),
    "yrtb_release_cached_memory": ([], ctypes.c_int),
    "yrtb_autotune": ([c_vp, c_vp, _P(yrtb_events), ctypes.c_int, c_u64,
                       _P(yrtb_tune_report), c_vp], ctypes.c_int),
    "yrtb_multiray_offsets": ([c_vp, c_u64, c_vp, c_vp], ctypes.c_int),
    "yrtb_multiray_table": ([c_vp, c_u64, c_vp], ctypes.c_int),
    "yrtb_forward": ([c_vp, c_vp, _P(yrtb_events), yrtb_range, c_vp, c_vp],
                     ctypes.c_int),
    "yrtb_backward": ([c_vp, c_vp, _P(yrtb_events), yrtb_range, c_vp, c_vp],
                      ctypes.c_int),
    "yrtb_em_step": ([c_vp, c_vp, c_vp, _P(yrtb_events), yrtb_range, c_f, c_f,
                      c_vp], ctypes.c_int),
    "yrtb_em_step_model": ([c_vp, c_vp, c_vp, _P(yrtb_events), yrtb_range, c_f, c_f,
                            c_vp, c_vp], ctypes.c_int),
    "yrtb_count_crossings": ([c_vp, _P(yrtb_events), yrtb_range, c_vp, c_vp],
                             ctypes.c_int),
    "yrtb_attenuation_factors": ([c_vp, c_vp, _P(yrtb_image_params),
                                  _P(yrtb_events), yrtb_range, c_vp, c_vp],
                                 ctypes.c_int),
    "yrtb_gather_histo3d": ([c_vp, c_vp, _P(yrtb_events), yrtb_range,
                             ctypes.c_int, c_vp, c_vp], ctypes.c_int),
    "yrtb_sensitivity_histo3d": ([c_vp, c_vp, c_vp, c_vp, c_vp,
                                  _P(yrtb_image_params), ctypes.c_int,
                                  ctypes.c_int, c_vp], ctypes.c_int),
    "yrtb_sensitivity_histo3d_crystal": ([c_vp, c_vp, c_vp, c_vp, c_vp,
                                          _P(yrtb_image_params), ctypes.c_int,
                                          ctypes.c_int, c_vp], ctypes.c_int),
    "yrtb_gather_crystal_product": ([c_vp, c_vp, _P(yrtb_events), yrtb_range,
                                     c_vp, c_vp], ctypes.c_int),
    "yrtb_em_step_histo3d": ([c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                              ctypes.c_int, ctypes.c_int, c_f, c_f, c_vp],
                             ctypes.c_int),
    "yrtb_histo3d_subset_nonzero": ([c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_u64,
                                     _P(c_u64), c_vp], ctypes.c_int),
    "yrtb_em_step_histo3d_list": ([c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                   ctypes.c_int, ctypes.c_int, c_vp, c_u64, c_f, c_f,
                                   c_vp], ctypes.c_int),
    "yrtb_listmode_to_histo3d": ([c_vp, c_vp, c_vp, c_vp, c_u64, c_vp,
                                  _P(c_u64), c_vp], ctypes.c_int),
    "yrtb_events_subset_order": ([c_vp, _P(yrtb_events), ctypes.c_int, c_vp,
                                  c_vp, c_vp], ctypes.c_int),
    "yrtb_events_subset_order_from": ([c_vp, _P(yrtb_events), ctypes.c_int, c_u64,
                                       c_vp, c_vp, c_vp], ctypes.c_int),
    "yrtb_events_gather": ([_P(yrtb_events), c_vp, _P(yrtb_events), c_vp],
                           ctypes.c_int),
    "yrtb_events_from_rows": ([c_vp, c_u64, _P(yrtb_row_layout), _P(yrtb_events),
                               c_vp], ctypes.c_int),
    "yrtb_unpack_listmode": ([c_vp, c_u64, ctypes.c_int, ctypes.c_int,
                              ctypes.c_uint32, c_vp, c_vp, c_vp, c_vp, c_vp,
                              c_vp], ctypes.c_int),
    "yrtb_histo3d_bins": ([c_vp, c_vp, c_vp, c_u64, c_vp, c_vp], ctypes.c_int),
    "yrtb_histo3d_detpairs": ([c_vp, c_vp, c_u64, c_vp, c_vp, c_vp],
                              ctypes.c_int),
    "yrtb_em_update": ([c_vp, c_vp, c_vp, c_u64, c_i64, c_i64, c_f, c_vp,
                        c_vp], ctypes.c_int),
    "yrtb_apply_threshold": ([c_vp, c_vp, c_u64, c_i64, ctypes.c_int, c_f, c_f,
                              c_f, c_f, c_f, c_vp], ctypes.c_int),
    "yrtb_fill": ([c_vp, c_u64, c_f, c_vp], ctypes.c_int),
    "yrtb_scale": ([c_vp, c_u64, c_f, c_vp], ctypes.c_int),
    "yrtb_lr_expand": ([c_vp, c_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, c_vp, c_vp],
                       ctypes.c_int),
    "yrtb_lr_contract_w": ([c_vp, c_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, c_vp,
                            c_vp], ctypes.c_int),
    "yrtb_lr_contract_h": ([c_vp, c_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, c_vp,
                            c_vp], ctypes.c_int),
    "yrtb_lr_update_h": ([c_vp, c_vp, c_vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, c_vp],
                         ctypes.c_int),
    "yrtb_varpsf_gaussian_kernel": ([c_vp, ctypes.c_int, c_vp, _P(yrtb_image_params), c_vp,
                                     ctypes.c_uint64, c_vp, c_vp], ctypes.c_int),
    "yrtb_varpsf_create": ([c_vp, c_vp, ctypes.c_int, c_vp, c_vp, _P(c_vp)], ctypes.c_int),
    "yrtb_varpsf_destroy": ([c_vp], None),
    "yrtb_varpsf_apply": ([c_vp, c_vp, c_vp, _P(yrtb_image_params), ctypes.c_int, c_vp],
                          ctypes.c_int),
    "yrtb_psf_create": ([c_vp, ctypes.c_int, c_vp, ctypes.c_int, c_vp, ctypes.c_int,
                         _P(c_vp)], ctypes.c_int),
    "yrtb_psf_destroy": ([c_vp], None),
    "yrtb_psf_apply": ([c_vp, c_vp, c_vp, _P(yrtb_image_params), ctypes.c_int, c_vp,
                        c_vp], ctypes.c_int),
    "yrtb_osem_listmode": ([c_vp, _P(yrtb_events), c_vp, c_vp, c_vp,
                            _P(yrtb_osem_params), c_vp], ctypes.c_int),
    "yrtb_osem_listmode_static": ([c_vp, _P(yrtb_events), c_vp, c_vp,
                                   _P(yrtb_osem_params), c_vp], ctypes.c_int),
}

_lib = None


class YrtbError(RuntimeError):
    """Raised for every non-zero status of the C ABI (the reference raises
    std::runtime_error / std::range_error, seen as RuntimeError in Python)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[yrtb error {code}] {msg}")
        self.code = code


def lib():
    """The loaded libyrtb.so; raises if it is absent (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libyrtb.so not found at {LIB_PATH}: build it with "
                "`python yrt-pet_b200/build.py` (CUDA path required)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int):
    if status != YRTB_OK:
        raise YrtbError(status, lib().yrtb_last_error().decode())
