"""Low-rank dynamic reconstruction mirroring the reference LREM / LREM_GPU
(src/recon/LREM.cpp, src/recon/LREM_GPU.cu) and the LR projector updater
(src/operators/ProjectorUpdater.cpp:228-280,
include/yrt-pet/operators/ProjectorUpdaterDevice.cuh:53-225).

The dynamic image is x_t = sum_l H[l][t] W_l: W holds `rank` images, H is
rank x frames (HBasis).  The reference applies the rank sum at every voxel
crossing (rank gathers forward, rank atomics backward).  Here each subset
expands the frames once (yrtb_lr_expand), runs the frame-indexed EM kernel on
them (one gather and one atomic per crossing), and contracts the
frame-indexed EM image onto W (yrtb_lr_contract_w) or H (yrtb_lr_contract_h).
The expanded frames are bit-identical to the values the reference's updater
forms at each crossing.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .core import DeviceProjector, ListModeLUT, _dev, _stream
from .osem import OSEM_GPU

UPDATER_TYPES = ("DEFAULT4D", "LR", "LRDUALUPDATE")


def _check(t: torch.Tensor, n: int, dtype=torch.float32):
    if not (t.is_cuda and t.dtype == dtype and t.is_contiguous() and t.numel() == n):
        raise RuntimeError("expected a contiguous CUDA tensor of %d %s" % (n, dtype))


def lr_expand(W: torch.Tensor, H: torch.Tensor, out: Optional[torch.Tensor] = None):
    """Frames X[t] = sum_l W[l] H[l][t] (W: (rank, ...) images, H: rank x T)."""
    R, T = H.shape
    J = W.numel() // R
    _check(W, R * J)
    _check(H, R * T)
    if out is None:
        out = torch.empty((T,) + tuple(W.shape[1:]), dtype=torch.float32, device=W.device)
    _check(out, T * J)
    L.check(L.lib().yrtb_lr_expand(W.data_ptr(), H.data_ptr(), R, T, J, out.data_ptr(),
                                   _stream()))
    return out


def lr_contract_w(E: torch.Tensor, H: torch.Tensor, out: Optional[torch.Tensor] = None):
    """Wn[l] = sum_t H[l][t] E[t] (E: (T, ...) frame images)."""
    R, T = H.shape
    J = E.numel() // T
    _check(E, T * J)
    _check(H, R * T)
    if out is None:
        out = torch.empty((R,) + tuple(E.shape[1:]), dtype=torch.float32, device=E.device)
    _check(out, R * J)
    L.check(L.lib().yrtb_lr_contract_w(E.data_ptr(), H.data_ptr(), R, T, J, out.data_ptr(),
                                       _stream()))
    return out


def lr_contract_h(W: torch.Tensor, E: torch.Tensor, rank: int,
                  out: Optional[torch.Tensor] = None):
    """Hn[l][t] = sum_j W[l][j] E[t][j] in FP64 (deterministic)."""
    J = W.numel() // rank
    T = E.numel() // J
    _check(W, rank * J)
    _check(E, T * J)
    if out is None:
        out = torch.empty((rank, T), dtype=torch.float64, device=W.device)
    _check(out, rank * T, torch.float64)
    L.check(L.lib().yrtb_lr_contract_h(W.data_ptr(), E.data_ptr(), rank, T, J,
                                       out.data_ptr(), _stream()))
    return out


def lr_update_h(H: torch.Tensor, Hn: torch.Tensor, c: torch.Tensor, eps: float):
    """H[r][t] *= float(Hn[r][t]) / max(c[r], eps)  (LREM::applyHUpdate)."""
    R, T = H.shape
    _check(H, R * T)
    _check(Hn, R * T, torch.float64)
    _check(c, R)
    L.check(L.lib().yrtb_lr_update_h(H.data_ptr(), Hn.data_ptr(), c.data_ptr(), R, T,
                                     float(eps), _stream()))
    return H


def w_update_scaling(H: np.ndarray) -> np.ndarray:
    """c_r = sum_t H[r][t], summed in FP32 in t order
    (LREM::generateWUpdateSensScaling, src/recon/LREM.cpp:201-218)."""
    H = np.ascontiguousarray(H, np.float32)
    out = np.zeros(H.shape[0], np.float32)
    for r in range(H.shape[0]):
        acc = np.float32(0)
        for v in H[r]:
            acc = np.float32(acc + v)
        out[r] = acc
    return out


class LowRankProjector:
    """Forward / back projection of a low-rank image through a frame-indexed
    DeviceProjector (its image has nt = frames; events carry their dynamic
    frame): the LR updater of OperatorProjectorDevice."""

    def __init__(self, proj: DeviceProjector, H):
        self.proj = proj
        self.H = _dev(H, torch.float32).contiguous()
        R, T = self.H.shape
        if proj.img_params.nt != T:
            raise RuntimeError("the projector's frames must match HBasis columns")

    def forward(self, W: torch.Tensor, ev, out=None, rng=None):
        X = lr_expand(W.contiguous(), self.H)
        return self.proj.forward(X, ev, out=out, rng=rng)

    def backward(self, values: torch.Tensor, ev, rng=None):
        E = self.proj.backward(values, ev, rng=rng)
        return lr_contract_w(E, self.H)

    def backward_h(self, values: torch.Tensor, W: torch.Tensor, ev, rng=None):
        """Back projection onto the temporal basis: Hn[l][t] =
        sum over events of frame t, voxels j of value * weight * W[l][j]."""
        E = self.proj.backward(values, ev, rng=rng)
        return lr_contract_h(W.contiguous(), E, self.H.shape[0])


class LREM_GPU(OSEM_GPU):
    """Low-rank list-mode EM (createOSEM(scanner, True, isLowRank=True)).
    setHBasis / setHBasisFromNumpy bind a rank x frames float32 array; with
    setUpdateH(True) the reconstruction updates H in that array (W fixed),
    otherwise it updates W (the returned rank images) with H fixed."""

    def __init__(self, scanner):
        super().__init__(scanner)
        self.projectorParams.updaterType = "LR"
        self._H: Optional[np.ndarray] = None
        self.projectorParams.updateH = False

    # ------------------------------------------------------------ LREM API --
    def isLowRank(self) -> bool:
        return self.projectorParams.updaterType in ("LR", "LRDUALUPDATE")

    def isDualUpdate(self) -> bool:
        return self.projectorParams.updaterType == "LRDUALUPDATE"

    def setUpdateH(self, update_h: bool):
        self.projectorParams.updateH = bool(update_h)

    def setHBasis(self, h_basis):
        self.setHBasisFromNumpy(h_basis)

    def setHBasisFromNumpy(self, h_basis):
        h = h_basis
        if not isinstance(h, np.ndarray) or h.ndim != 2:
            raise RuntimeError("HBasis must be 2D (rank x time).")
        if h.dtype != np.float32:
            raise RuntimeError("HBasis must be float32.")
        if not h.flags["C_CONTIGUOUS"]:
            raise RuntimeError("HBasis must be C-contiguous.")
        self._H = h  # bound, not copied: an H update writes into it

    def getHBasisNumpy(self) -> np.ndarray:
        if self._H is None or self._H.size == 0:
            raise RuntimeError("HBasis not set (empty alias)")
        return self._H.copy()

    def setProjectorUpdaterType(self, updater_type):
        name = getattr(updater_type, "name", str(updater_type)).upper()
        if name not in UPDATER_TYPES:
            raise RuntimeError("Projector updater type not valid")
        self.projectorParams.updaterType = name

    def getProjectorUpdaterType(self) -> str:
        return self.projectorParams.updaterType

    # ----------------------------------------------------------- reconstruct --
    def reconstruct(self, out_fname: str = "") -> torch.Tensor:
        if not self.isLowRank():
            return super().reconstruct(out_fname)
        if self.isDualUpdate():
            raise RuntimeError("LRDUALUPDATE updater is not implemented on GPU yet")
        if self._H is None:
            raise RuntimeError("The H matrix is not defined. Impossible to do "
                               "Low-Rank reconstruction.")
        if self._data is None:
            raise RuntimeError("Data input unspecified")
        if not self._sens_images:
            raise RuntimeError("Sensitivity image(s) not set")
        if self.num_OSEM_subsets <= 0 or self.num_MLEM_iterations <= 0:
            raise RuntimeError("Not enough OSEM subsets / MLEM iterations")
        if self.imageParams is None:
            raise RuntimeError("Image parameters not valid/set")
        if not self.usingListModeInput or not isinstance(self._data, ListModeLUT):
            raise RuntimeError("low-rank reconstruction needs list-mode input "
                               "with dynamic framing")
        if self.flagImagePSF:
            raise RuntimeError("image-space PSF is not supported with the "
                               "low-rank updater")
        return self._reconstruct_lr()

    def _reconstruct_lr(self) -> torch.Tensor:
        lm: ListModeLUT = self._data
        Hh = self._H
        R, T = Hh.shape
        if lm.getNumDynamicFrames() != T:
            raise RuntimeError(
                f"HBasis has {T} frames but the list-mode has "
                f"{lm.getNumDynamicFrames()} dynamic frames")
        update_h = bool(self.projectorParams.updateH)
        ipX = self.imageParams.withFrames(T)
        J = ipX.numVoxels
        proj = DeviceProjector(self.scanner, ipX, self.projectorParams)
        ev, offsets = self._listmode_events(
            proj, lm, self.num_OSEM_subsets if self.orderEvents else 0)
        lib = L.lib()
        st = _stream()
        nsub = self.num_OSEM_subsets
        # List-mode sensitivity, shared by the subsets and divided by their
        # number (OSEM::initializeSensImageBuffer).
        sens = self._sens_images[0].reshape(-1)[:J]
        sens_sub = sens.clone()
        if nsub != 1:
            L.check(lib.yrtb_scale(sens_sub.data_ptr(), J,
                                   float(np.float32(1) / np.float32(nsub)), st))
        # W: initial estimate or 0.125, masked by the sensitivity (or mask).
        W = torch.empty(R * J, dtype=torch.float32, device="cuda")
        if self._initial is not None:
            W.copy_(_dev(self._initial, torch.float32).reshape(-1))
        else:
            L.check(lib.yrtb_fill(W.data_ptr(), W.numel(), self.INITIAL_VALUE_MLEM, st))
        mask = self._mask.reshape(-1) if self._mask is not None else sens
        L.check(lib.yrtb_apply_threshold(W.data_ptr(), mask.data_ptr(), J, R, 1,
                                         0.0, 0.0, 0.0, 1.0, 0.0, st))
        H = torch.from_numpy(Hh).cuda().contiguous()
        if update_h:
            cH64 = lr_contract_h(W, sens_sub, R)
            c = cH64.reshape(R).to(torch.float32).contiguous()
        else:
            c = torch.from_numpy(w_update_scaling(Hh)).cuda()
        X = torch.empty(T * J, dtype=torch.float32, device="cuda")
        E = torch.empty(T * J, dtype=torch.float32, device="cuda")
        Wn = None if update_h else torch.empty(R * J, dtype=torch.float32, device="cuda")
        Hn = torch.empty((R, T), dtype=torch.float64, device="cuda") if update_h else None
        evc = ev.c()
        for it in range(self.num_MLEM_iterations):
            for s in range(nsub):
                if offsets is None:
                    r = L.yrtb_range(s, nsub, 0)
                else:
                    r = L.yrtb_range(int(offsets[s]), 1, int(offsets[s + 1] - offsets[s]))
                lr_expand(W, H, out=X)
                E.zero_()
                if offsets is None or r.count:
                    L.check(lib.yrtb_em_step(proj.h, X.data_ptr(), E.data_ptr(),
                                             ctypes.byref(evc), r, float(self._global),
                                             float(self.denomThreshold), st))
                if update_h:
                    lr_contract_h(W, E, R, out=Hn)
                    lr_update_h(H, Hn, c, self.EPS_FLT)
                else:
                    lr_contract_w(E, H, out=Wn)
                    L.check(lib.yrtb_em_update(W.data_ptr(), Wn.data_ptr(),
                                               sens_sub.data_ptr(), J, R, 1,
                                               self.EPS_FLT, c.data_ptr(), st))
            # The MLEM image of the low-rank updater is W (R basis images).
            self._save_iteration(it, W, self.imageParams.withFrames(R).shape)
        if update_h:
            Hh[...] = H.cpu().numpy()
        self._last_events = ev
        return W.reshape(self.imageParams.withFrames(R).shape)
