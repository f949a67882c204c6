"""Per-configuration benchmark runs behind `bench.py --config c1|c3|c4|c5`.

The default `bench.py` line is the C2 workload (50M TOF events).  These runs
measure the other four configurations of the projection path on one GPU,
each printing one JSON line:

  c1  list-mode OSEM, Siddon without TOF, 16 rings x 256 crystals, 128x128x64
      image, 1M events: sensitivity image (8.32M-bin uniform histogram) and
      2 iterations x 5 subsets; reference CPU OSEM on the same events and the
      image difference.
  c3  list-mode -> Histogram3D binning of 200M events (bit-exact check on a
      sample against the reference), then histogram-mode OSEM with the
      distance-driven projector and a 4 mm FWHM projection-space PSF,
      200x200x100 image at 2.5 mm, 3 iterations x 12 subsets.
  c4  differentiable TOF Siddon: Poisson log-likelihood and its gradient for
      8 phantoms x 5M TOF events (forward + adjoint per phantom).
  c5  24 dynamic frames with per-frame rigid motion on the C2 scanner and
      image (1.0 GB 4D image), frame sizes log-uniform in [2e5, 2e7]:
      batched form (all frames in one EM launch per subset, CUDA-graph
      subsets) against the plain form (one single-frame reconstruction per
      frame).
  psf image-space PSF (applyA + applyAH) on the C2 image, bit-exact against
      the reference operator.
  lrem low-rank list-mode EM (rank 8, 20 frames) on the C2 scanner and image,
      20M TOF events: per-stage times of expand / EM pass / contraction.

Inputs are seeded synthetic events (the reference's datasets are not
available); the reference CPU measurements use oracle/_ref, the reference
library built from its sources, where present.
"""
from __future__ import annotations

import ctypes
import json
import os
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))


def _yrt():
    sys.path.insert(0, os.path.join(ROOT, "yrt-pet_b200"))
    import pyyrtpet_b200 as yrt
    from pyyrtpet_b200 import _lib as L
    from pyyrtpet_b200 import synthetic as S
    from pyyrtpet_b200.core import _stream
    return yrt, L, S, _stream


def _po():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    return po


class Timer:
    """CUDA-event timer on the current stream."""

    def __enter__(self):
        torch.cuda.synchronize()
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)
        self.a.record()
        return self

    def __exit__(self, *exc):
        self.b.record()
        torch.cuda.synchronize()
        self.ms = self.a.elapsed_time(self.b)
        return False


def _po_scanner(po, sc):
    return po.Scanner(sc.axialFOV, sc.crystalSize_z, sc.crystalSize_trans,
                      sc.crystalDepth, sc.scannerRadius, sc.detsPerRing,
                      sc.numRings, sc.numDOI, sc.maxRingDiff, sc.minAngDiff,
                      sc.detsPerBlock)


def _po_image(po, ip, nt=1):
    return po.ImageParams(ip.nx, ip.ny, ip.nz, ip.length_x, ip.length_y,
                          ip.length_z, nt=nt)


def _rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _roofline(launch, alg_bytes, kernel, per_unit, reps=5):
    """Roofline of the dominant kernel of a configuration: its algorithmic
    bytes per launch (alg_bytes, stated by the caller from the per-unit
    figures in per_unit) over its CUDA-event time on the launching stream
    (median of reps launches after two warm-up launches), against the HBM
    peak (measured, else the fallback, as bench.py)."""
    import bench
    for _ in range(2):
        launch()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        launch()
        b.record(st)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    ms = float(np.median(ts))
    peak, kind = bench.measured_peak_hbm()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": kind, "traffic": None,
            "kernel": kernel, "alg_bytes_per_launch": float(alg_bytes),
            "alg_bytes_per_unit": per_unit, "kernel_ms_per_launch": ms}


def _visits(proj, ev, rng=None):
    """Voxel visits (crossings or footprint voxels, all rays) of the events
    of rng, and the number of those events."""
    c = proj.count_crossings(ev, rng).double()
    if rng is None or rng.count == 0:
        return float(c.sum().item()), int(ev.count)
    return float(c.sum().item()), int(rng.count)


def _base(cfg, metric, value, unit, steps, warmup, ms, config):
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": 1,
            "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded phantom events)",
            "config": dict(workload=cfg, **config)}


# ------------------------------------------------------------------- C1 ----
def run_c1(args):
    """List-mode OSEM, Siddon without TOF, C1 scanner/image, 1M events."""
    yrt, L, S, _stream = _yrt()
    sc = S.scanner_c1()
    ip = S.image_c1()
    ev = S.generate_events(sc, 1_000_000, 20261203 + 0, device="cuda",
                           chunk=1 << 24)
    e = {"d1": ev.d1.cpu().numpy().astype(np.uint32),
         "d2": ev.d2.cpu().numpy().astype(np.uint32)}
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 2
    osem.num_OSEM_subsets = 5
    osem.setListModeEnabled(True)
    for _ in range(args.warmup):
        osem.generateSensitivityImages()
    with Timer() as ts:
        sens = osem.generateSensitivityImages()
    lm = yrt.ListModeLUT(sc)
    lm.bind(e["d1"], e["d2"])
    osem.setDataInput(lm)
    # Launch configuration: tuned once on subset 0 (set-up, not timed), then
    # reused by the timed reconstructions.
    osem.autotune = True
    osem.reconstruct()
    osem.launchConfig = osem.lastTuneReport["best"]
    osem.autotune = False
    for _ in range(args.warmup):
        osem.reconstruct()
    times = []
    img = None
    for _ in range(args.steps):
        with Timer() as t:
            img = osem.reconstruct()
        times.append(t.ms)
    ms = float(np.median(times))
    out = _base("C1 list-mode OSEM 2x5, Siddon, no TOF, 16x256 scanner, "
                "128x128x64 @2mm, 1M events",
                "events/s (list-mode OSEM, Siddon, events x iterations / time)",
                1e6 * 2 / (ms * 1e-3), "events/s", args.steps, args.warmup, ms,
                {"events": 1_000_000, "iterations": 2, "subsets": 5,
                 "launch": osem.launchConfig})
    out["sens_image_ms"] = ts.ms
    out["sens_bins"] = int(yrt.Histogram3D(sc).count())
    # Roofline of the fused EM kernel over subset 0 (the reconstruction's own
    # projector parameters, launch configuration and event order).
    rp = yrt.DeviceProjector(sc, ip, osem.projectorParams)
    rp.set_launch(**osem.launchConfig)
    dev = yrt.DeviceEvents.from_arrays(torch.from_numpy(e["d1"].view(np.int32)).cuda(),
                                       torch.from_numpy(e["d2"].view(np.int32)).cuda())
    dev, offs = rp.order_events(dev, 5)
    r0 = L.yrtb_range(int(offs[0]), 1, int(offs[1] - offs[0]))
    nv, ne = _visits(rp, dev, r0)
    x0 = torch.full((ip.numVoxels,), 0.125, device="cuda")
    em0 = torch.zeros_like(x0)
    out["roofline"] = _roofline(
        lambda: rp.em_step(x0, em0, dev, rng=r0), 8 * ne + 12 * nv,
        "k_events<OP_EM, K_SIDDON, mirror> (fused fwd->ratio->bwd, subset 0)",
        {"per_event": "8 B (d1, d2)", "per_crossing": "12 B (4 B gather, 8 B reduction)",
         "events": ne, "crossings": nv})
    po = _po()
    if po.ref_available() and not args.no_cpu_baseline:
        osc = _po_scanner(po, sc)
        oip = _po_image(po, ip)
        rs, rsec = po.ref_sensitivity(osc, oip, listmode=True,
                                      threads=os.cpu_count() or 1)
        rimg, rosec = po.ref_osem_listmode(osc, oip, rs[0], e["d1"], e["d2"],
                                           iterations=2, subsets=5,
                                           threads=os.cpu_count() or 1)
        out["cpu_baseline"] = {
            "value": 1e6 * 2 / rosec, "unit": "events/s",
            "cores": os.cpu_count(), "kind": "reference",
            "sample": "the full workload (1M events, 2 x 5)",
            "sens_image_s": rsec, "osem_s": rosec}
        out["parity_vs_reference"] = {
            "sens_rel_l2": _rel_l2(sens[0].cpu().numpy(), rs[0]),
            "image_rel_l2": _rel_l2(img.cpu().numpy(), rimg)}
    return out


# ------------------------------------------------------------------- C5 ----
def run_c5(args):
    """24 dynamic frames with rigid motion: batched vs plain single-frame."""
    yrt, L, S, _stream = _yrt()
    sc = S.scanner_c2()
    ip1 = S.image_c2()
    nt = 24
    subsets = 10
    counts = S.frame_counts_loguniform(nt, 2e5, 2e7, 20261203 + 4)
    if args.cfg_events:
        counts = np.maximum(1, np.round(counts * (args.cfg_events / counts.sum()))).astype(np.int64)
    n = int(counts.sum())
    ev = S.generate_events(sc, n, 20261203 + 4, tof_fwhm_ps=214.0, device="cuda",
                           chunk=1 << 24)
    frames = torch.repeat_interleave(torch.arange(nt, device="cuda", dtype=torch.int32),
                                     torch.from_numpy(counts).cuda())
    motion = S.rigid_transforms(nt, 20261203 + 5)
    ipT = ip1.withFrames(nt)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = L.YRTB_COMPENSATED
    proj = yrt.DeviceProjector(sc, ipT, pp)
    d1 = ev.d1.to(torch.int32)
    d2 = ev.d2.to(torch.int32)
    base = yrt.DeviceEvents.from_arrays(d1, d2, tof=ev.tof, frame=frames,
                                        motion_frame=frames, motion=motion)
    J = ip1.numVoxels
    sens_proj = yrt.DeviceProjector(sc, ip1, yrt.ProjectorParams(sc))
    sens = torch.zeros(J, device="cuda")
    for part in range(20):  # all bins of the histogram, in 20 parts
        sens_proj.sensitivity_histo3d(sens, 20, part)
    s_ptr = _stream()
    lib = L.lib()
    # The reference's hard threshold (1.0) on the sensitivity image.
    L.check(lib.yrtb_apply_threshold(sens.data_ptr(), sens.data_ptr(), J, 1, 1,
                                     1.0, 0.0, 0.0, 1.0, 0.0, s_ptr))

    # Batched: one event set for all frames, subset-major / frame ordering,
    # one CUDA graph per subset replayed by yrtb_osem_listmode; launch
    # configuration from the autotuner (set-up, not timed).
    probe = torch.full((nt * ip1.numVoxels,), 0.125, device="cuda")
    tune = proj.autotune(probe, base, subsets)
    del probe
    ordered, offs = proj.order_events(base, subsets)
    evc = ordered.c()
    img = torch.empty(nt * J, device="cuda")
    work = torch.empty((nt + 1) * J, device="cuda")
    stream = torch.cuda.Stream()

    def batched(iters):
        p = L.yrtb_osem_params(iters, subsets, 1.0, 1e-35, 1.19209e-07, 0, 1,
                               None, offs.ctypes.data)
        with torch.cuda.stream(stream):
            L.check(lib.yrtb_osem_listmode(proj.h, ctypes.byref(evc),
                                           sens.data_ptr(), img.data_ptr(),
                                           work.data_ptr(), ctypes.byref(p),
                                           _stream()))
        torch.cuda.current_stream().wait_stream(stream)

    # Plain: one single-frame reconstruction per frame (events in file order,
    # interleaved subsets), as a frame-by-frame reference workflow runs it.
    proj1 = yrt.DeviceProjector(sc, ip1, pp)
    starts = np.concatenate([[0], np.cumsum(counts)])
    per_frame = []
    for f in range(nt):
        a, b = int(starts[f]), int(starts[f + 1])
        per_frame.append(yrt.DeviceEvents.from_arrays(
            d1[a:b], d2[a:b], tof=ev.tof[a:b],
            motion_frame=torch.full((b - a,), f, dtype=torch.int32, device="cuda"),
            motion=motion))
    img1 = torch.empty(J, device="cuda")
    work1 = torch.empty(2 * J, device="cuda")

    def plain(iters):
        p = L.yrtb_osem_params(iters, subsets, 1.0, 1e-35, 1.19209e-07, 0, 0,
                               None, None)
        for f in range(nt):
            L.check(lib.yrtb_osem_listmode(proj1.h, ctypes.byref(per_frame[f].c()),
                                           sens.data_ptr(), img1.data_ptr(),
                                           work1.data_ptr(), ctypes.byref(p),
                                           s_ptr))

    for _ in range(max(1, args.warmup)):
        batched(1)
        plain(1)
    bt, pt = [], []
    for _ in range(args.steps):
        # NVTX ranges let a profiler select the timed launches of each form.
        torch.cuda.nvtx.range_push("c5_batched")
        with Timer() as t:
            batched(1)
        torch.cuda.nvtx.range_pop()
        bt.append(t.ms)
        torch.cuda.nvtx.range_push("c5_plain")
        with Timer() as t:
            plain(1)
        torch.cuda.nvtx.range_pop()
        pt.append(t.ms)
    ms_b = float(np.median(bt))
    ms_p = float(np.median(pt))
    out = _base("C5 dynamic + motion list-mode TOF OSEM, 24 frames (log-uniform "
                "2e5-2e7 events), C2 scanner/image, 10 subsets",
                "events/s (one OSEM iteration over all frames, batched)",
                n / (ms_b * 1e-3), "events/s", args.steps, args.warmup, ms_b,
                {"events": n, "frames": nt, "subsets": subsets,
                 "precision": "compensated", "launch": tune["best"]})
    out["plain"] = {"value": n / (ms_p * 1e-3), "ms_per_step": ms_p,
                    "what": "24 separate single-frame reconstructions (one per "
                            "frame, file order, interleaved subsets)"}
    out["batched_over_plain"] = ms_p / ms_b
    out["frame_events"] = [int(c) for c in counts]
    # Roofline of the batched EM kernel over subset 0 (all frames' events).
    r0 = L.yrtb_range(int(offs[0]), 1, int(offs[1] - offs[0]))
    nv, ne = _visits(proj, ordered, r0)
    x0 = torch.full((nt * J,), 0.125, device="cuda")
    em0 = torch.zeros_like(x0)
    out["roofline"] = _roofline(
        lambda: proj.em_step(x0, em0, ordered, rng=r0), 20 * ne + 12 * nv,
        "k_events<OP_EM, K_SIDDON, TOF, compensated> over all 24 frames (subset 0)",
        {"per_event": "20 B (d1, d2, TOF, frame, motion frame)",
         "per_crossing": "12 B (4 B gather, 8 B reduction)", "events": ne,
         "crossings": nv})
    if not args.no_cpu_baseline:
        out.update(_c5_reference(args, sc, ip1, nt, subsets, counts, d1, d2, ev.tof,
                                 motion, sens, n / (ms_b * 1e-3)))
    return out


def _c5_reference(args, sc, ip1, nt, subsets, counts, d1, d2, tof, motion, sens,
                  batched_value):
    """The reference on the C5 workload (events/s of one OSEM iteration):
    its CPU OSEM with DynamicFraming and LORMotion on a 2M-event sample
    (frame shares kept), and its GPU OSEM_GPU (built for sm_100a) on all
    events, both as one 4-D reconstruction and frame by frame (24 separate
    single-frame reconstructions: the plain single-frame GPU form)."""
    po = _po()
    threads = os.cpu_count() or 1
    out = {}
    osc = _po_scanner(po, sc)
    J = ip1.numVoxels
    sens_np = sens.reshape(ip1.nz, ip1.ny, ip1.nx).cpu().numpy()
    h1 = d1.cpu().numpy().view(np.uint32)
    h2 = d2.cpu().numpy().view(np.uint32)
    ht = tof.cpu().numpy()
    starts = np.concatenate([[0], np.cumsum(counts)])
    frame_ts = (np.arange(nt + 1) * 1000).astype(np.uint32)
    motion_starts = (np.arange(nt) * 1000).astype(np.uint32)
    kw = dict(tof_fwhm_ps=214.0, tof_n_std=5, iterations=1, subsets=subsets,
              threads=threads)
    if po.ref_available():
        # Sample: the first events of every frame, in the frames' proportions.
        share = 2_000_000 / float(counts.sum())
        take = np.maximum(1, np.round(counts * share)).astype(np.int64)
        idx = np.concatenate([np.arange(starts[f], starts[f] + take[f]) for f in range(nt)])
        ts = (np.repeat(np.arange(nt), take) * 1000 + 500).astype(np.uint32)
        _, sec = po.ref_osem_listmode_dynamic(
            osc, _po_image(po, ip1, nt=nt), sens_np, h1[idx], h2[idx], ts,
            frame_ts=frame_ts, motion_starts=motion_starts, motion=motion,
            tof=ht[idx], gpu=False, **kw)
        out["cpu_baseline"] = {"value": len(idx) / sec, "unit": "events/s",
                               "cores": threads, "kind": "reference",
                               "sample": f"{len(idx)} events (every frame's first "
                                         "events, frame shares kept), one OSEM "
                                         f"iteration x {subsets} subsets with "
                                         "DynamicFraming and LORMotion"}
    if po.ref_gpu_available():
        ts_all = (np.repeat(np.arange(nt), counts) * 1000 + 500).astype(np.uint32)
        _, sec4 = po.ref_osem_listmode_dynamic(
            osc, _po_image(po, ip1, nt=nt), sens_np, h1, h2, ts_all,
            frame_ts=frame_ts, motion_starts=motion_starts, motion=motion,
            tof=ht, gpu=True, **kw)
        total = 0.0
        for f in range(nt):
            a, b = int(starts[f]), int(starts[f + 1])
            _, secf = po.ref_osem_listmode_dynamic(
                osc, _po_image(po, ip1, nt=1), sens_np, h1[a:b], h2[a:b],
                np.full(b - a, 500, np.uint32),
                frame_ts=np.array([0, 1000], np.uint32),
                motion_starts=np.array([0], np.uint32), motion=motion[f:f + 1],
                tof=ht[a:b], gpu=True, **kw)
            total += secf
        n = int(counts.sum())
        out["plain_reference_gpu"] = {
            "value": n / total, "unit": "events/s", "s_per_iteration": total,
            "what": "reference OSEM_GPU (YRT-PET built for sm_100a) frame by "
                    "frame: 24 single-frame reconstructions of one iteration, "
                    "OSEM::reconstruct time summed"}
        out["reference_gpu_4d"] = {
            "value": n / sec4, "unit": "events/s", "s_per_iteration": sec4,
            "what": "reference OSEM_GPU, one 4-D reconstruction of all frames "
                    "(DynamicFraming + LORMotion), one iteration"}
        out["batched_vs_plain_reference_gpu"] = batched_value / (n / total)
    return out


def _gaussian_psf(fwhm=4.0, ks=0.5):
    sig = fwhm / 2.3548
    half = int(np.ceil(3 * sig / ks))
    x = (np.arange(2 * half + 1) - half) * ks
    k = np.exp(-0.5 * (x / sig) ** 2)
    k /= k.sum() * ks
    return 1e9, ks, k[None].astype(np.float32)


# ------------------------------------------------------------------- C3 ----
def run_c3(args):
    """200M events -> Histogram3D; DD + projection PSF histogram OSEM."""
    import tempfile
    yrt, L, S, _stream = _yrt()
    sc = S.scanner_c1(15)
    ip = S.image_c3()
    total = args.cfg_events or 200_000_000
    chunk = 20_000_000
    h = yrt.Histogram3D(sc)
    hist = torch.zeros(h.histoSize, dtype=torch.float32, device="cuda")
    p0 = yrt.core._scratch_projector(sc)
    bin_ms = 0.0
    sample = None
    done = 0
    seed = 20261203 + 3
    while done < total:
        m = min(chunk, total - done)
        ev = S.generate_events(sc, m, seed + done, device="cuda", chunk=1 << 24)
        a = ev.d1.to(torch.int32).contiguous()
        b = ev.d2.to(torch.int32).contiguous()
        if sample is None:
            sample = (a[:2_000_000].cpu().numpy().view(np.uint32),
                      b[:2_000_000].cpu().numpy().view(np.uint32))
        bad = ctypes.c_uint64()
        with Timer() as t:
            L.check(L.lib().yrtb_listmode_to_histo3d(
                p0.h, a.data_ptr(), b.data_ptr(), None, m, hist.data_ptr(),
                ctypes.byref(bad), _stream()))
        bin_ms += t.ms
        done += m
        del ev, a, b
    h.data = hist.cpu().numpy()
    s_step, ks, taps = _gaussian_psf()
    csv = os.path.join(tempfile.mkdtemp(), "psf.csv")
    yrt.write_psf_csv(csv, s_step, ks, taps)
    osem = yrt.createOSEM(sc)
    osem.setImageParams(ip)
    osem.num_MLEM_iterations = 3
    osem.num_OSEM_subsets = 12
    osem.setProjector("DD")
    osem.addProjPSF(csv)
    # Compensated precision: PSF integrals from prefix sums.
    osem.projectorParams.precision = L.YRTB_COMPENSATED
    osem.setDataInput(h)
    with Timer() as ts:
        sens = osem.generateSensitivityImages()
    osem.num_MLEM_iterations = 1
    for _ in range(args.warmup):
        osem.reconstruct()
    times = []
    for _ in range(args.steps):
        with Timer() as t:
            img = osem.reconstruct()
        times.append(t.ms)
    ms = float(np.median(times))
    nz = int((hist > 0).sum().item())
    out = _base("C3 histogram OSEM, distance-driven + projection PSF (4 mm FWHM), "
                "C1 scanner mrd 15 (8.32M bins) from 200M events, 200x200x100 "
                "@2.5mm, 12 subsets",
                "histogram bins/s (DD+PSF OSEM iteration over all bins)",
                h.count() / (ms * 1e-3), "bins/s", args.steps, args.warmup, ms,
                {"events_binned": total, "bins": h.count(), "nonzero_bins": nz,
                 "subsets": 12, "precision": "compensated"})
    out["binning"] = {"events_per_s": total / (bin_ms * 1e-3), "ms": bin_ms}
    out["sens_images_ms"] = ts.ms
    out["osem_s_per_iteration"] = ms * 1e-3
    # Roofline of the histogram EM kernel over subset 0's list of non-zero
    # bins (the reconstruction's projector parameters).
    rp = yrt.DeviceProjector(sc, ip, osem.projectorParams)
    it = yrt.BinIteratorRangeHistogram3D(h.numZBin, h.numPhi, h.numR, 12, 0)
    bins0 = rp.histo3d_subset_nonzero(hist, 12, 0, it.size())
    glob = it.indices()[bins0.cpu().numpy()].astype(np.uint64)
    pa, pb = yrt.histo3d_detpairs(sc, glob)
    nv, nb = _visits(rp, yrt.DeviceEvents.from_arrays(pa, pb))
    x0 = torch.full((ip.numVoxels,), 0.125, device="cuda")
    em0 = torch.zeros_like(x0)
    out["roofline"] = _roofline(
        lambda: rp.em_step_histo3d(x0, em0, hist, 12, 0, bins=bins0), 12 * nb + 12 * nv,
        "k_histo<K_DD_PSF, EM, compensated, 4 threads per bin> (subset 0's non-zero bins)",
        {"per_bin": "12 B (measurement, list entry)",
         "per_footprint_voxel": "12 B (4 B gather, 8 B reduction)", "bins": nb,
         "footprint_voxels": nv})
    po = _po()
    if po.ref_available() and not args.no_cpu_baseline:
        osc = _po_scanner(po, sc)
        ours = yrt.ListModeLUT(sc)
        ours.bind(*sample)
        mine = yrt.convertToHistogram3D(ours).data
        ref_h, ref_s = po.ref_lm_to_histo3d(osc, *sample, threads=os.cpu_count() or 1)
        out["binning"]["bitexact_vs_reference_2M_sample"] = bool(
            np.array_equal(mine.view(np.uint32), ref_h.view(np.uint32)))
        out["binning"]["reference_events_per_s"] = len(sample[0]) / ref_s
        oip = _po_image(po, ip)
        rimg, rsec = po.ref_osem_histo3d(osc, oip,
                                         np.stack([x.cpu().numpy() for x in sens]),
                                         h.data, psf_csv=csv, projector="DD",
                                         iterations=1, subsets=12,
                                         threads=os.cpu_count() or 1)
        out["cpu_baseline"] = {"value": h.count() / rsec, "unit": "bins/s",
                               "cores": os.cpu_count(), "kind": "reference",
                               "sample": "1 OSEM iteration x 12 subsets of the "
                                         "same histogram"}
        out["parity_vs_reference"] = {"image_rel_l2_1_iteration": _rel_l2(
            img.cpu().numpy(), rimg)}
    return out


# ------------------------------------------------------------------- C4 ----
def run_c4(args):
    """Poisson NLL + gradient through the autograd projector, 8 phantoms."""
    yrt, L, S, _stream = _yrt()
    from pyyrtpet_b200.autograd import poisson_nll, poisson_nll_fused
    sc = S.scanner_c1()
    ip = S.image_c1()
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = L.YRTB_COMPENSATED
    proj = yrt.DeviceProjector(sc, ip, pp)
    per = (args.cfg_events or 40_000_000) // 8
    evs, imgs = [], []
    for b in range(8):
        ph = S.random_phantom(20261203 + 40 + b, sc.axialFOV / 2)
        e = S.generate_events(sc, per, 20261203 + 40 + b, phantom=ph,
                              tof_fwhm_ps=214.0, device="cuda", chunk=1 << 24)
        evs.append(yrt.DeviceEvents.from_arrays(e.d1.to(torch.int32),
                                                e.d2.to(torch.int32), tof=e.tof))
        imgs.append(ph.image(ip, device="cuda") + 0.1)
    x = torch.stack(imgs).contiguous().requires_grad_(True)
    sens = torch.ones(ip.shape, device="cuda")
    # Set-up (not timed): launch configuration from the autotuner, then each
    # phantom's events in the tuned order (the loss does not depend on it).
    tune = proj.autotune(x[0].detach().contiguous(), evs[0], 1)
    evs = [proj.order_events(e, 1)[0] for e in evs]

    def step(fn):
        x.grad = None
        loss = fn(x, proj, evs, sens).sum()
        loss.backward()
        return loss

    def timed(fn):
        for _ in range(args.warmup):
            step(fn)
        times = []
        for _ in range(args.steps):
            with Timer() as t:
                step(fn)
            times.append(t.ms)
        return float(np.median(times))

    # Fused: loss and gradient from one EM-kernel pass per phantom
    # (PoissonNLLFn); composed: the projector's autograd Function (forward
    # kernel, torch reductions, adjoint kernel in backward).
    ms = timed(poisson_nll_fused)
    ms_c = timed(poisson_nll)
    out = _base("C4 differentiable TOF Siddon: Poisson NLL + gradient, 8 "
                "phantoms x 5M TOF events, C1 scanner, 128x128x64 @2mm",
                "events/s (forward + adjoint per event, autograd)",
                per * 8 / (ms * 1e-3), "events/s", args.steps, args.warmup, ms,
                {"phantoms": 8, "events_per_phantom": per,
                 "precision": "compensated", "launch": tune["best"],
                 "loss": "PoissonNLLFn (one fused pass per phantom)"})
    out["composed"] = {"value": per * 8 / (ms_c * 1e-3), "ms_per_step": ms_c,
                       "what": "SiddonProjectFn forward kernel + torch FP64 reductions + "
                               "adjoint kernel in backward"}
    # Roofline of the fused pass of one phantom (loss terms and gradient).
    ev0 = evs[0]
    x0 = x[0].detach().contiguous()
    em0 = torch.zeros_like(x0)
    model = torch.empty(ev0.count, device="cuda")
    nv, ne = _visits(proj, ev0)
    out["roofline"] = _roofline(
        lambda: proj.em_step(x0, em0, ev0, model=model), 16 * ne + 12 * nv,
        "k_events<OP_EM, K_SIDDON, TOF, compensated> writing the model (one phantom)",
        {"per_event": "16 B (d1, d2, TOF, model value)",
         "per_crossing": "12 B (4 B gather, 8 B reduction)", "events": ne,
         "crossings": nv})
    po = _po()
    if po.ref_available() and not args.no_cpu_baseline:
        # The reference CPU forward + back projection (util::forwProject /
        # util::backProject) of the first phantom's first 1M events, TOF.
        m = min(per, 1_000_000)
        osc = _po_scanner(po, sc)
        oip = _po_image(po, ip)
        e0 = evs[0]
        a = e0.d1[:m].cpu().numpy().view(np.uint32)
        b = e0.d2[:m].cpu().numpy().view(np.uint32)
        tv = e0.tof[:m].cpu().numpy()
        xv = x[0].detach().cpu().numpy()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        yv = po.ref_project_lm(osc, oip, a, b, tof=tv, image=xv, tof_fwhm_ps=214.0,
                               tof_n_std=5, threads=threads)
        w = np.where(yv > 1e-12, 1.0 / np.maximum(yv, 1e-12), 0.0).astype(np.float32)
        po.ref_project_lm(osc, oip, a, b, tof=tv, values=w, fwd=False,
                          tof_fwhm_ps=214.0, tof_n_std=5, threads=threads)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": m / sec, "unit": "events/s",
                               "cores": threads, "kind": "reference",
                               "sample": f"{m} events of phantom 0: forward "
                                         "projection, 1/y, back projection "
                                         "(util::forwProject + util::backProject)"}
    return out


# ------------------------------------------------------- image-space PSF --
def run_psf(args):
    """Image-space PSF (OperatorPsfDevice applyA + applyAH) on the C2 image,
    4 mm FWHM Gaussian; bit-exact check and CPU time of the reference
    operator on the same image."""
    yrt, L, S, _stream = _yrt()
    ip = S.image_c2()
    psf = yrt.OperatorPsfDevice.createGaussianFromFWHM(4.0, 4.0, 4.0, ip.vx, ip.vy, ip.vz)
    g = torch.Generator(device="cuda").manual_seed(20261203)
    x = torch.rand(ip.shape, generator=g, device="cuda")
    a = torch.empty_like(x)
    ah = torch.empty_like(x)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    V = ip.numVoxels

    def step():
        psf.applyA(x, a, ip)
        psf.applyAH(a, ah, ip)

    for _ in range(args.warmup):
        step()
    resident, cold = [], []
    for _ in range(args.steps):
        with Timer() as t:
            step()
        resident.append(t.ms)
        flush.fill_(1)
        with Timer() as t:
            step()
        cold.append(t.ms)
    ms_res = float(np.median(resident))
    ms_cold = float(np.median(cold))
    # Three passes per apply, each reading and writing every voxel once.
    alg = 2 * 3 * 8 * V
    peaks = _measured_peaks()
    out = _base("image-space PSF (separable 3-D convolution, circular borders), "
                "C2 image 256x256x160 @2mm, 4 mm FWHM Gaussian (5 taps per axis)",
                "voxels/s (applyA + applyAH per voxel)", V / (ms_res * 1e-3),
                "voxels/s", args.steps, args.warmup, ms_res,
                {"kernel_taps": [len(psf.getKernelX()), len(psf.getKernelY()),
                                 len(psf.getKernelZ())],
                 "image_bytes": 4 * V, "l2": "image L2-resident (42 MB); "
                 "cold = after a 256 MB flush"})
    out["roofline"] = {"bound": "hbm", "achieved": alg / (ms_cold * 1e-3) / 1e9,
                       "peak": peaks, "unit": "GB/s",
                       "frac": alg / (ms_cold * 1e-3) / 1e9 / peaks,
                       "traffic": None, "note": "cold (flushed) step; 48 B/voxel "
                       "algorithmic (3 passes x 2 applies x read + write)"}
    out["ms_per_step_cold"] = ms_cold
    po = _po()
    if po.ref_available():
        host = x.cpu().numpy()
        oip = _po_image(po, ip)
        t0 = time.perf_counter()
        ref = po.ref_psf_convolve(oip, host, psf.getKernelX(), psf.getKernelY(),
                                  psf.getKernelZ())
        ref = po.ref_psf_convolve(oip, ref, psf.getKernelX(), psf.getKernelY(),
                                  psf.getKernelZ(), adjoint=True)
        sec = time.perf_counter() - t0
        out["bitexact_vs_reference"] = bool(np.array_equal(
            ref.view(np.uint32), ah.cpu().numpy().view(np.uint32)))
        out["cpu_baseline"] = {"value": V / sec, "unit": "voxels/s", "cores": 1,
                               "kind": "reference",
                               "sample": "the same image, applyA + applyAH "
                               "(OperatorPsf, single-threaded)"}
    out["variant"] = _run_varpsf(args, yrt, ip, x, po)
    return out


def _run_varpsf(args, yrt, ip, x, po):
    """Spatially variant PSF on the same image: 5 x 5 x 5 Gaussian LUT over
    200 mm in 50 mm steps, 4 sigmas, sigmas 1.2-1.8 mm (3 or 5 taps per axis)."""
    import tempfile
    rng = np.random.default_rng(20261203 + 70)
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        f.write("200,200,200\n50,50,50\n4,4,4\n")
        for _ in range(125):
            f.write(",".join("%.6g" % v for v in rng.uniform(1.2, 1.8, 3)) + "\n")
        csv = f.name
    op = yrt.OperatorVarPsfDevice(csv, ip)
    a = torch.empty_like(x)
    ah = torch.empty_like(x)
    for _ in range(args.warmup):
        op.applyA(x, a)
        op.applyAH(x, ah)
    fwd, adj = [], []
    for _ in range(args.steps):
        with Timer() as t:
            op.applyA(x, a)
        fwd.append(t.ms)
        with Timer() as t:
            op.applyAH(x, ah)
        adj.append(t.ms)
    res = {"lut": "5x5x5 Gaussian kernels, sigma 1.2-1.8 mm, 4 sigmas",
           "applyA_ms": float(np.median(fwd)), "applyAH_ms": float(np.median(adj)),
           "voxels_per_s_applyA": ip.numVoxels / (np.median(fwd) * 1e-3)}
    if po.ref_available():
        host = x.cpu().numpy()
        t0 = time.perf_counter()
        ref = po.ref_varpsf_apply(_po_image(po, ip), csv, host, threads=os.cpu_count() or 1)
        sec = time.perf_counter() - t0
        res["applyA_bitexact_vs_reference"] = bool(np.array_equal(
            ref.view(np.uint32), a.cpu().numpy().view(np.uint32)))
        res["cpu_baseline"] = {"value": ip.numVoxels / sec, "unit": "voxels/s (applyA)",
                               "cores": os.cpu_count() or 1, "kind": "reference",
                               "sample": "the same image, OperatorVarPsf::applyA"}
    os.unlink(csv)
    return res


# ---------------------------------------------------------- low-rank EM ----
def run_lrem(args):
    """Low-rank list-mode EM (W update): rank 8, 20 dynamic frames, C2 scanner
    and image, 20M TOF events spread evenly over the frames, 4 subsets."""
    yrt, L, S, _stream = _yrt()
    from pyyrtpet_b200 import lrem
    sc = S.scanner_c2()
    ip1 = S.image_c2()
    R, T, subsets = 8, 20, 4
    n = args.cfg_events or 20_000_000
    ev = S.generate_events(sc, n, 20261203 + 60, tof_fwhm_ps=214.0, device="cuda",
                           chunk=1 << 24)
    frames = ((torch.arange(n, device="cuda", dtype=torch.int64) * T) // n).to(torch.int32)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(214.0, 5)
    pp.precision = L.YRTB_COMPENSATED
    ipT = ip1.withFrames(T)
    proj = yrt.DeviceProjector(sc, ipT, pp)
    base = yrt.DeviceEvents.from_arrays(ev.d1.to(torch.int32), ev.d2.to(torch.int32),
                                        tof=ev.tof, frame=frames)
    J = ip1.numVoxels
    sens_proj = yrt.DeviceProjector(sc, ip1, yrt.ProjectorParams(sc))
    sens = torch.zeros(J, device="cuda")
    for part in range(20):  # all bins of the histogram, in 20 parts
        sens_proj.sensitivity_histo3d(sens, 20, part)
    lib = L.lib()
    st = _stream()
    g = torch.Generator(device="cuda").manual_seed(20261203 + 61)
    H = (0.2 + torch.rand((R, T), generator=g, device="cuda")).contiguous()
    c = torch.from_numpy(lrem.w_update_scaling(H.cpu().numpy())).cuda()
    sens_sub = (sens * np.float32(1.0 / subsets)).contiguous()
    X = torch.empty(T * J, device="cuda")
    E = torch.empty(T * J, device="cuda")
    Wn = torch.empty(R * J, device="cuda")
    W = torch.full((R * J,), 0.125, device="cuda")
    # Set-up (not timed): launch configuration and subset-major event order.
    lrem.lr_expand(W, H, out=X)
    tune = proj.autotune(X, base, subsets)
    ordered, offs = proj.order_events(base, subsets)
    evc = ordered.c()
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    stage = np.zeros(4)

    def subset(sidx, record):
        r = L.yrtb_range(int(offs[sidx]), 1, int(offs[sidx + 1] - offs[sidx]))
        if record:
            marks[0].record()
        lrem.lr_expand(W, H, out=X)
        if record:
            marks[1].record()
        E.zero_()
        L.check(lib.yrtb_em_step(proj.h, X.data_ptr(), E.data_ptr(), ctypes.byref(evc), r,
                                 1.0, 1e-35, st))
        if record:
            marks[2].record()
        lrem.lr_contract_w(E, H, out=Wn)
        if record:
            marks[3].record()
        L.check(lib.yrtb_em_update(W.data_ptr(), Wn.data_ptr(), sens_sub.data_ptr(), J, R,
                                   1, 1.19209e-07, c.data_ptr(), st))
        if record:
            marks[4].record()

    def step(record=False):
        for sidx in range(subsets):
            subset(sidx, record)
            if record:
                torch.cuda.synchronize()
                for k in range(4):
                    stage[k] += marks[k].elapsed_time(marks[k + 1])

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        with Timer() as t:
            step()
        times.append(t.ms)
    stage[:] = 0
    step(record=True)
    per_subset = stage / subsets
    ms = float(np.median(times))
    out = _base("low-rank list-mode EM (W update), rank 8 x 20 frames, C2 scanner "
                "80x672, 256x256x160 @2mm, 20M TOF events, 4 subsets",
                "events/s (one EM iteration over all events, low-rank image)",
                n / (ms * 1e-3), "events/s", args.steps, args.warmup, ms,
                {"rank": R, "frames": T, "subsets": subsets, "events": n,
                 "precision": "compensated", "launch": tune["best"],
                 "l2": "expanded frames 840 MB and rank images 336 MB exceed L2"})
    peaks = _measured_peaks()
    # expand: read R, write T images; contract: read T, write R images.
    bytes_expand = 4.0 * J * (R + T)
    bytes_contract = 4.0 * J * (T + R)
    out["stages_ms_per_subset"] = {"expand": per_subset[0], "em_pass": per_subset[1],
                                   "contract_w": per_subset[2], "update": per_subset[3]}
    out["roofline"] = {"bound": "hbm",
                       "achieved": bytes_expand / (per_subset[0] * 1e-3) / 1e9,
                       "peak": peaks, "unit": "GB/s",
                       "frac": bytes_expand / (per_subset[0] * 1e-3) / 1e9 / peaks,
                       "traffic": None,
                       "note": "yrtb_lr_expand: 4 (R + T) B per voxel; contract_w "
                               "achieves %.0f GB/s" % (bytes_contract /
                                                        (per_subset[2] * 1e-3) / 1e9)}
    po = _po()
    if po.ref_available():
        m = 200_000
        d1 = ev.d1[:m].cpu().numpy().astype(np.uint32)
        d2 = ev.d2[:m].cpu().numpy().astype(np.uint32)
        tof = ev.tof[:m].cpu().numpy()
        ts = np.arange(m, dtype=np.uint32)
        fts = np.linspace(0, m, T + 1).astype(np.uint32)
        t0 = time.perf_counter()
        po.ref_lrem_listmode(_po_scanner(po, sc), _po_image(po, ip1, nt=R),
                             sens.cpu().numpy(), d1, d2, ts, fts,
                             H.cpu().numpy(), tof=tof, iterations=1, subsets=1,
                             tof_fwhm_ps=214.0, tof_n_std=5,
                             threads=os.cpu_count() or 1)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": m / sec, "unit": "events/s",
                               "cores": os.cpu_count() or 1, "kind": "reference",
                               "sample": "200k events of the workload, 1 iteration, "
                                         "1 subset, LREM_CPU (wall time incl. set-up)"}
    return out


def _measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


# ------------------------------------------------------ C2 multi-ray ----
def run_c2mr(args):
    """The C2 TOF list-mode workload with 4-ray Siddon (rays after the first
    offset across the crystal faces, curand stream per event): one OSEM
    iteration x 10 subsets through yrtb_osem_listmode, beside the same
    iteration with one ray, the reference CPU 4-ray OSEM on a sample, and
    the 4-ray forward projections of a sample against the FP64 oracle with
    the device's ray offsets."""
    import bench
    yrt, L, S, _stream = _yrt()
    n = args.cfg_events or bench.NUM_EVENTS
    sc, ip, ph, eff, evs, mu = bench.build_workload(n, "cuda", seed=bench.SEED)
    mu_flat = mu.reshape(-1).contiguous()
    J = ip.numVoxels
    # Sensitivity image (set-up, not timed): all histogram bins, attenuation
    # from the mu-map.
    sens_proj = yrt.DeviceProjector(sc, ip, yrt.ProjectorParams(sc))
    sens = torch.zeros(J, device="cuda")
    for part in range(20):
        sens_proj.sensitivity_histo3d(sens, 20, part, mu=mu_flat, mu_params=ip)
    lib = L.lib()
    n_rand_lors = float(sc.getNumDets()) ** 2 / 2 * 0.45
    ms = {}
    proj4 = None
    # 4 rays with one lane per ray (the default), 4 rays with one thread
    # walking them in turn, and one ray.
    for rays, lanes in ((4, 4), (4, 1), (1, 1)):
        pp = yrt.ProjectorParams(sc)
        pp.addTOF(bench.TOF_FWHM, bench.TOF_NSTD)
        pp.numRays = rays
        pp.precision = L.YRTB_COMPENSATED
        proj = yrt.DeviceProjector(sc, ip, pp)
        if rays == 4:
            cfg = proj.get_launch()
            cfg["threads_per_lor"] = lanes
            if lanes > 1 and getattr(args, "vector_groups", -1) >= 0:
                cfg["vector_groups"] = args.vector_groups
            proj.set_launch(**cfg)
        if rays == 4 and lanes == 4:
            proj4 = proj
        ev = yrt.DeviceEvents.from_arrays(evs.d1.to(torch.int32), evs.d2.to(torch.int32),
                                          tof=evs.tof)
        ev, offs = proj.order_events(ev, bench.SUBSETS)
        ev.sens = (eff[ev.d1.long()] * eff[ev.d2.long()]).contiguous()
        ev.att = proj.attenuation_factors(mu_flat, ip, ev)
        ev.additive = torch.full((ev.count,), 0.2 * ev.count / n_rand_lors, device="cuda")
        if rays > 1:
            # Set-up, not timed: the offsets of every item index of a subset.
            with Timer() as tt:
                proj.multiray_table(int(np.max(np.diff(offs))))
            table_ms = tt.ms
        img = torch.empty(J, device="cuda")
        work = torch.empty(2 * J, device="cuda")
        p = L.yrtb_osem_params(1, bench.SUBSETS, 1.0, 1e-35, 1.19209e-07, 0, 0, None,
                               offs.ctypes.data)

        def one():
            L.check(lib.yrtb_osem_listmode(proj.h, ctypes.byref(ev.c()), sens.data_ptr(),
                                           img.data_ptr(), work.data_ptr(),
                                           ctypes.byref(p), _stream()))
        for _ in range(max(1, args.warmup)):
            one()
        times = []
        for _ in range(args.steps):
            with Timer() as t:
                one()
            times.append(t.ms)
        ms[(rays, lanes)] = float(np.median(times))
        if rays == 4 and lanes == 4:
            # Roofline of the 4-ray EM kernel over subset 0.
            r0 = L.yrtb_range(int(offs[0]), 1, int(offs[1] - offs[0]))
            nv, ne = _visits(proj, ev, r0)
            x0 = torch.full((J,), 0.125, device="cuda")
            em0 = torch.zeros_like(x0)
            roof = _roofline(
                lambda: proj.em_step(x0, em0, ev, rng=r0), 24 * ne + 12 * nv,
                "k_events<OP_EM, K_SIDDON_MR, TOF, compensated, one lane per ray> (subset 0)",
                {"per_event": "24 B (d1, d2, TOF, sens, att, additive)",
                 "per_crossing": "12 B (4 B gather, 8 B reduction), 4 rays",
                 "events": ne, "crossings": nv})
            del x0, em0
        del ev, img, work
    out = _base("C2 list-mode TOF OSEM iteration with 4-ray Siddon, 80x672 scanner "
                "R=410, 256x256x160 @2mm, 214 ps TOF 5 sigma, 10 subsets",
                "events/s (4-ray fwd+back TOF Siddon, one OSEM iteration)",
                n / (ms[(4, 4)] * 1e-3), "events/s", args.steps, args.warmup, ms[(4, 4)],
                {"events": n, "rays": 4, "subsets": bench.SUBSETS,
                 "precision": "compensated",
                 "multi_ray_stream": "curand XORWOW, seed 13, subsequence = event "
                                     "index in the call"})
    out["single_ray"] = {"value": n / (ms[(1, 1)] * 1e-3), "ms_per_step": ms[(1, 1)]}
    out["one_thread_per_event"] = {"value": n / (ms[(4, 1)] * 1e-3),
                                   "ms_per_step": ms[(4, 1)],
                                   "what": "4 rays walked in turn by one thread per event"}
    out["cost_vs_single_ray"] = ms[(4, 4)] / ms[(1, 1)]
    out["roofline"] = roof
    out["launch"] = proj4.get_launch()
    out["multiray_table_ms"] = table_ms
    # FP64 parity of the 4-ray forward projections on a sample, with the
    # offsets the device draws for it.
    po = _po()
    k = 20000
    d1 = evs.d1[:k].to(torch.int32).cpu().numpy().view(np.uint32)
    d2 = evs.d2[:k].to(torch.int32).cpu().numpy().view(np.uint32)
    tof = evs.tof[:k].cpu().numpy()
    g = torch.Generator(device="cuda").manual_seed(20261203 + 21)
    x = (0.5 + torch.rand(ip.shape, generator=g, device="cuda")).contiguous()
    v = proj4.forward(x, yrt.DeviceEvents.from_arrays(d1, d2, tof=tof)).cpu().numpy()
    roffs = proj4.multiray_offsets(k).cpu().numpy()
    lors, ori = po.lors_from_detpairs(po.scanner_lut(_po_scanner(po, sc)), d1, d2)
    ref = po.project(_po_image(po, ip),
                     po.Proj(num_rays=4, crystal_z=sc.crystalSize_z,
                             crystal_trans=sc.crystalSize_trans,
                             tof_fwhm_ps=bench.TOF_FWHM, tof_n_std=bench.TOF_NSTD),
                     lors, image=x.cpu().numpy(), orients=ori, tof=tof, ray_offsets=roffs,
                     precision="f64")
    out["parity_vs_fp64"] = {"fwd_rel_l2": _rel_l2(v, ref), "sample_events": k}
    if po.ref_available() and not args.no_cpu_baseline:
        m = 200_000
        osc = _po_scanner(po, sc)
        oip = _po_image(po, ip)
        _, sec = po.ref_osem_listmode(
            osc, oip, np.ones((ip.nz, ip.ny, ip.nx), np.float32),
            evs.d1[:m].cpu().numpy().astype(np.uint32),
            evs.d2[:m].cpu().numpy().astype(np.uint32),
            tof=evs.tof[:m].cpu().numpy().astype(np.float32),
            randoms=np.full(m, 1e-3, np.float32), att_params=oip,
            att_image=mu.cpu().numpy(), iterations=1, subsets=bench.SUBSETS,
            tof_fwhm_ps=bench.TOF_FWHM, tof_n_std=bench.TOF_NSTD, num_rays=4,
            threads=os.cpu_count() or 1)
        out["cpu_baseline"] = {"value": m / sec, "unit": "events/s",
                               "cores": os.cpu_count(), "kind": "reference",
                               "sample": f"{m} events of the workload, one 4-ray OSEM "
                                         "iteration x 10 subsets (includes the "
                                         "reference's correction precompute)"}
    return out


# ------------------------------------------------------- walk sequences ----
def run_walks(args):
    """Voxel index sequences of the single-ray Siddon walks on the first
    events of the C2 workload (yrtb_trace_walks, LOR input), against the CPU
    restatement's FP32 and FP64 walks (orc_siddon_trace_f32/_f64): the
    number of rays whose offset sequences differ, per precision mode, without
    and with TOF.  A parity measurement, not a timing."""
    import bench
    yrt, L, S, _stream = _yrt()
    po = _po()
    n = args.cfg_events or 20000
    sc, ip, ph, eff, evs, mu = bench.build_workload(n, "cuda")
    d1 = evs.d1.cpu().numpy().astype(np.uint32)
    d2 = evs.d2.cpu().numpy().astype(np.uint32)
    tof = evs.tof.cpu().numpy()
    lors, _ = po.lors_from_detpairs(po.scanner_lut(bench.ref_scanner(po, sc)), d1, d2)
    oip = _po_image(po, ip)
    out = {"metric": "voxel index sequences of the Siddon walks vs the CPU restatement",
           "config": {"workload": "C2 scanner and image, the first events of the bench "
                                  "workload", "events": n}}
    for tof_on in (False, True):
        pr = po.Proj(tof_fwhm_ps=bench.TOF_FWHM if tof_on else 0.0,
                     tof_n_std=bench.TOF_NSTD if tof_on else 0)
        ev = yrt.DeviceEvents.from_arrays(lor=lors, tof=tof if tof_on else None)
        seq = {}
        for prec in (L.YRTB_MIRROR, L.YRTB_COMPENSATED):
            pp = yrt.ProjectorParams(sc)
            if tof_on:
                pp.addTOF(bench.TOF_FWHM, bench.TOF_NSTD)
            pp.precision = prec
            o, w, c = yrt.DeviceProjector(sc, ip, pp).trace_walks(ev, 1024)
            o, c = o.cpu().numpy(), c.cpu().numpy()
            seq[prec] = [o[k, :c[k]] for k in range(n)]
        f32 = [po.siddon_trace(oip, pr, lors[k], float(tof[k]))[0] for k in range(n)]
        f64 = [po.siddon_trace_f64(oip, pr, lors[k], float(tof[k]))[0] for k in range(n)]

        def differ(a, b):
            return int(sum(not np.array_equal(x, y) for x, y in zip(a, b)))
        m, cmp = seq[L.YRTB_MIRROR], seq[L.YRTB_COMPENSATED]
        out["tof" if tof_on else "non_tof"] = {
            "rays": n, "mirror_vs_fp32_restatement": differ(m, f32),
            "mirror_vs_fp64": differ(m, f64), "compensated_vs_fp64": differ(cmp, f64),
            "compensated_vs_mirror": differ(cmp, m),
            "mean_crossings": float(np.mean([len(x) for x in m]))}
    return out


RUNNERS = {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5,
           "psf": run_psf, "lrem": run_lrem, "c2mr": run_c2mr, "walks": run_walks}
