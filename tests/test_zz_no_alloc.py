"""yrtb_osem_listmode_static: list-mode OSEM for callers that cannot allocate
device memory (their host owns all device memory through its own pool, or
forbids cudaMalloc/cudaFree -- which synchronise the device -- once running).

The entry point keeps its scratch in one static device array, so it takes no
work buffer.  It must give the same image as yrtb_osem_listmode with a
caller-provided work buffer (tolerance: rel-L2 1e-5, the run-to-run spread of
the float atomics), also on a second call in a row that reuses the array.

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import pyyrtpet_b200 as yrt
from pyyrtpet_b200 import _lib as L
from pyyrtpet_b200 import synthetic as S
from pyyrtpet_b200.core import _stream

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = a.double().ravel()
    b = b.double().ravel()
    return float((a - b).norm() / b.norm())


def _problem(nx=64, ny=64, nz=32):
    sc = S.scanner_c1()
    ip = yrt.ImageParams(nx, ny, nz, 256, 256, 128)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    proj = yrt.DeviceProjector(sc, ip, pp)
    evs = S.generate_events(sc, 60000, 31, tof_fwhm_ps=214.0, device="cuda")
    ev = yrt.DeviceEvents.from_arrays(evs.d1.to(torch.int32), evs.d2.to(torch.int32),
                                      tof=evs.tof)
    sens_proj = yrt.DeviceProjector(sc, ip, yrt.ProjectorParams(sc))
    sens = torch.zeros(ip.numVoxels, device="cuda")
    sens_proj.sensitivity_histo3d(sens, 1, 0)
    return ip, proj, ev, sens


def _params(use_graph=0):
    return L.yrtb_osem_params(2, 3, 1.0, 1e-35, 1.19209e-07, 0, use_graph,
                              None, None)


def test_static_osem_matches_work_buffer_osem_twice():
    ip, proj, ev, sens = _problem()
    J = ip.numVoxels
    evc = ev.c()
    p = _params()
    # Existing entry point, caller-provided work buffer.
    ref = torch.empty(J, device="cuda")
    work = torch.empty(2 * J, device="cuda")
    L.check(L.lib().yrtb_osem_listmode(proj.h, ctypes.byref(evc), sens.data_ptr(),
                                       ref.data_ptr(), work.data_ptr(),
                                       ctypes.byref(p), _stream()))
    # Allocation-free entry point, two calls in a row on the shared array.
    for _ in range(2):
        img = torch.empty(J, device="cuda")
        L.check(L.lib().yrtb_osem_listmode_static(
            proj.h, ctypes.byref(evc), sens.data_ptr(), img.data_ptr(),
            ctypes.byref(p), _stream()))
        torch.cuda.synchronize()
        assert torch.isfinite(img).all()
        assert rel_l2(img, ref) < 1e-5


def test_static_osem_allocates_nothing():
    # The property the entry point exists for: once the library's device
    # code is loaded (first call), a call changes neither the device's free
    # memory (cudaMemGetInfo: no cudaMalloc, no memory-pool growth) nor
    # torch's reserved memory.
    ip, proj, ev, sens = _problem(48, 48, 24)
    evc = ev.c()
    p = _params()
    img = torch.empty(ip.numVoxels, device="cuda")

    def call():
        L.check(L.lib().yrtb_osem_listmode_static(
            proj.h, ctypes.byref(evc), sens.data_ptr(), img.data_ptr(),
            ctypes.byref(p), _stream()))
        torch.cuda.synchronize()

    call()
    free0 = torch.cuda.mem_get_info()[0]
    reserved0 = torch.cuda.memory_reserved()
    call()
    call()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == reserved0
    assert torch.isfinite(img).all()


def test_static_osem_with_image_psf_matches_work_buffer_osem():
    # With an image-space PSF the scratch also holds the blurred image and
    # the PSF's temporary ((3 nt + 1) x voxels): same image as the work-buffer
    # driver given a (3 nt + 1) x voxels buffer, on two calls in a row.
    from pyyrtpet_b200 import OperatorPsfDevice
    ip, proj, ev, sens = _problem()
    J = ip.numVoxels
    k = np.array([0.25, 0.5, 0.25], np.float32)
    psf = OperatorPsfDevice(k, k, k)
    evc = ev.c()
    p = L.yrtb_osem_params(2, 3, 1.0, 1e-35, 1.19209e-07, 0, 0, None, None,
                           psf.handle, None)
    ref = torch.empty(J, device="cuda")
    work = torch.empty(4 * J, device="cuda")
    L.check(L.lib().yrtb_osem_listmode(proj.h, ctypes.byref(evc), sens.data_ptr(),
                                       ref.data_ptr(), work.data_ptr(),
                                       ctypes.byref(p), _stream()))
    for _ in range(2):
        img = torch.empty(J, device="cuda")
        L.check(L.lib().yrtb_osem_listmode_static(
            proj.h, ctypes.byref(evc), sens.data_ptr(), img.data_ptr(),
            ctypes.byref(p), _stream()))
        torch.cuda.synchronize()
        assert torch.isfinite(img).all()
        assert rel_l2(img, ref) < 1e-5


def test_static_osem_rejects_oversized_images_and_graphs():
    sc = S.scanner_c1()
    big = yrt.ImageParams(256, 256, 64, 256, 256, 128)   # 2 x 4.19M floats > 4M
    proj = yrt.DeviceProjector(sc, big, yrt.ProjectorParams(sc))
    ev = yrt.DeviceEvents.from_arrays(np.array([0], np.uint32),
                                      np.array([128], np.uint32))
    img = torch.zeros(big.numVoxels, device="cuda")
    sens = torch.ones(big.numVoxels, device="cuda")
    p = _params()
    rc = L.lib().yrtb_osem_listmode_static(proj.h, ctypes.byref(ev.c()),
                                           sens.data_ptr(), img.data_ptr(),
                                           ctypes.byref(p), _stream())
    assert rc == L.YRTB_ERR_ARGUMENT
    assert b"too large" in L.lib().yrtb_last_error()
    assert b"(3nt+1) x voxels with one" in L.lib().yrtb_last_error()
    small = yrt.ImageParams(16, 16, 8, 256, 256, 128)
    proj2 = yrt.DeviceProjector(sc, small, yrt.ProjectorParams(sc))
    pg = _params(use_graph=1)
    img2 = torch.zeros(small.numVoxels, device="cuda")
    sens2 = torch.ones(small.numVoxels, device="cuda")
    rc = L.lib().yrtb_osem_listmode_static(proj2.h, ctypes.byref(ev.c()),
                                           sens2.data_ptr(), img2.data_ptr(),
                                           ctypes.byref(pg), _stream())
    assert rc == L.YRTB_ERR_ARGUMENT
    assert b"use_graph" in L.lib().yrtb_last_error()
