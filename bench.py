#!/usr/bin/env python
"""Benchmark: list-mode TOF Siddon forward + back projection (fused OSEM EM
pass) on the 80-ring x 672-crystal scanner, 256x256x160 image at 2 mm, 50M
events with float32 TOF (214 ps FWHM, 5 sigma), lognormal crystal
efficiencies, water mu-map, 20 % uniform randoms; 10 subsets.

One step = one OSEM iteration: for each of the 10 subsets, clear the EM
image, run the fused forward -> ratio -> back projection over the subset's
5M events, and apply the multiplicative update.  `value` = events / s with
the events already resident in HBM; `e2e` = event-iterations / s of whole
reconstructions (3 iterations x 10 subsets) through the public OSEM API from
pinned host event arrays (H2D of the events, event ordering, correction
factors on device and D2H of the image inside the timed region).

Beside the timed line, on one GPU: the reference's own GPU reconstruction
(YRT-PET OSEM_GPU built for sm_100a from its sources) of the same 50M events
(`plain_reference_gpu`), the reference CPU reconstruction of a sample
(`cpu_baseline`), and the image error of this path against both
(`parity_vs_reference`).

    python bench.py [--gpus N] [--steps K] [--warmup W]
    python bench.py --impl reference     # reference CPU OSEM on a sample
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "yrt-pet_b200"))

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "events/s fwd+back TOF Siddon, batched vs plain on 1 GPU, rel err<1e-4 vs FP64"
UNIT = "events/s"
WORKLOAD = ("C2 list-mode TOF Siddon OSEM iteration (fused fwd+bwd), 80x672 scanner "
            "R=410, 256x256x160 @2mm, 214 ps TOF 5 sigma, 10 subsets")
NUM_EVENTS = 50_000_000
SUBSETS = 10
# OSEM iterations of one reconstruction of this workload (the end-to-end
# step and the reference arm run a whole reconstruction).
ITERATIONS = 3
TOF_FWHM = 214.0
TOF_NSTD = 5
SEED = 20261203 + 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--events", type=int, default=NUM_EVENTS)
    ap.add_argument("--ref-sample", type=int, default=1_000_000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the parity and reference legs")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference OSEM_GPU leg")
    ap.add_argument("--no-l2-peak", action="store_true",
                    help="skip the live L2 request-throughput measurement")
    ap.add_argument("--precision", default="compensated",
                    choices=["mirror", "compensated"])
    ap.add_argument("--parity-sample", type=int, default=200_000)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch configuration instead of "
                         "timing the candidates on a sample first")
    ap.add_argument("--tune-report", default="",
                    help="write every autotuner candidate and its time (JSON)")
    ap.add_argument("--deterministic", action="store_true",
                    help="two-pass fixed-point back projection")
    ap.add_argument("--vector-groups", type=int, default=-1,
                    help="force the launch's vector_groups after autotuning "
                         "(default: the autotuner's choice)")
    ap.add_argument("--layout", default="row", choices=["tile", "row"],
                    help="image layout of the timed EM passes: 4x2 tiles "
                         "(YRTB_LAYOUT_TILE_4X2) or the reference's row-major")
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c2mr", "c3", "c4", "c5", "psf", "lrem", "walks"],
                    help="c2 (default) is the headline workload; the others "
                         "run bench_configs.py")
    ap.add_argument("--cfg-events", type=int, default=0,
                    help="override the event count of --config c1/c2mr/c3/c4/c5/walks")
    return ap.parse_args()


# ----------------------------------------------------------------- workload --
def build_workload(n_events, device, seed=SEED, lut=None):
    """C2 scanner, image, phantom, crystal efficiencies, events, mu-map.
    lut (optional): the crystal LUT to use instead of this library's
    DetRegular LUT (the reference arm passes the reference's own, so that it
    never loads the product library; the two are bit-identical)."""
    from pyyrtpet_b200 import synthetic as S
    sc = S.scanner_c2()
    if lut is not None:
        sc.setDetectorLUT(lut)
    ip = S.image_c2()
    ph = S.Phantom(cyl_half_length=sc.axialFOV / 2)
    # One scanner for every shard: the efficiencies do not depend on the
    # events' seed.
    eff = S.crystal_efficiencies(sc, SEED + 1, device=device)
    ev = S.generate_events(sc, n_events, seed, phantom=ph, tof_fwhm_ps=TOF_FWHM,
                           mu_per_mm=0.0096, crystal_eff=eff,
                           randoms_fraction=0.2, device=device)
    mu = ph.mu_image(ip, device=device)
    return sc, ip, ph, eff, ev, mu


def additive_per_event(sc, n_events):
    """Flat randoms estimate per event: 20 % of the prompts spread uniformly
    over the LORs (about 45 % of all crystal pairs have a histogram bin)."""
    n_rand_lors = float(sc.getNumDets()) ** 2 / 2 * 0.45
    return 0.2 * n_events / n_rand_lors


def common_config(world, n_events, sample_events):
    """The workload as both arms state it (identical dicts)."""
    return {"workload": WORKLOAD, "events_per_gpu": n_events,
            "subsets": SUBSETS, "iterations_per_reconstruction": ITERATIONS,
            "corrections": "LOR sensitivity eff1*eff2 (lognormal crystal "
                           "efficiencies, sigma 0.1), attenuation from the "
                           "water mu-map, flat 20 % randoms estimate per event",
            "sensitivity_image": "all 1.44e9 Histogram3D bins, eff1*eff2 and "
                                 "attenuation, hard threshold 1.0",
            "sample_events": sample_events,
            "l2": "event arrays (1.2 GB) larger than L2; image (42 MB) "
                  "L2-resident by design",
            "parallelism": f"dp{world} (events sharded, EM image all-reduced "
                           "per subset)"}


def ref_scanner(po, sc):
    return po.Scanner(sc.axialFOV, sc.crystalSize_z, sc.crystalSize_trans,
                      sc.crystalDepth, sc.scannerRadius, sc.detsPerRing,
                      sc.numRings, sc.numDOI, sc.maxRingDiff, sc.minAngDiff,
                      sc.detsPerBlock)


def ref_image(po, ip):
    return po.ImageParams(ip.nx, ip.ny, ip.nz, ip.length_x, ip.length_y,
                          ip.length_z)


def loaded_libraries():
    """Shared libraries of this repository mapped into this process."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            path = line.split()[-1] if len(line.split()) >= 6 else ""
            if path.endswith(".so") and path.startswith(ROOT):
                out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def clocks_sampler(path):
    try:
        return subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader",
             "-lms", "200"], stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def summarize_clocks(path, gpu_index):
    sm, mx, reasons = [], None, set()
    try:
        for line in open(path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or f[0] != str(gpu_index):
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown",
                                "sw_thermal_slowdown", "sw_power_cap"], f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
    except OSError:
        pass
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons)}
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


L2_MODES = {0: "red.f32", 1: "red.v4.f32", 2: "ld.cg.f32",
            3: "ld.cg.f32 + red.v4.f32 (every warp)",
            4: "ld.cg.f32 + red.v4.f32 (reading warps beside reducing warps)"}


def measured_l2_request_rates(n_floats, reps=5):
    """L2 request throughput of this GPU (requests/s), measured live with
    libyrtb_l2bench.so: uniformly random aligned float groups inside two
    L2-resident buffers of n_floats each (the sizes of the image read and of
    the EM image reduced into), per request kind (L2_MODES), median of reps
    launches timed with CUDA events after warm-up."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "yrt-pet_b200", "lib", "libyrtb_l2bench.so"))
    lib.yrtb_l2bench_launch.restype = ctypes.c_int
    lib.yrtb_l2bench_launch.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_uint, ctypes.c_void_p,
                                        ctypes.c_void_p]
    lib.yrtb_l2bench_requests.restype = ctypes.c_uint64
    lib.yrtb_l2bench_requests.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint]
    n = 2 * ((int(n_floats) // 4) * 4)
    buf = torch.zeros(n, dtype=torch.float32, device="cuda")
    sink = torch.zeros(1, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    blocks = torch.cuda.get_device_properties(0).multi_processor_count * 8
    iters = 96
    out = {}
    for mode in L2_MODES:
        times = []
        for r in range(reps + 2):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            rc = lib.yrtb_l2bench_launch(buf.data_ptr(), n, mode, iters, blocks,
                                         sink.data_ptr(), st.cuda_stream)
            b.record(st)
            if rc != 0:
                raise RuntimeError(f"yrtb_l2bench_launch: error {rc}")
            torch.cuda.synchronize()
            if r >= 2:
                times.append(a.elapsed_time(b))
        ms = sorted(times)[len(times) // 2]
        out[L2_MODES[mode]] = lib.yrtb_l2bench_requests(mode, iters, blocks) / (ms * 1e-3)
    del buf, sink
    return out


# ------------------------------------------------------------ reference legs --
def reference_osem(po, sc, ip, d1, d2, tof, additive, sens, sens_histo, mu_np,
                   threads, gpu):
    """One reconstruction (ITERATIONS x SUBSETS) of the given events with the
    reference library: OSEM_CPU (oracle/_ref), or OSEM_GPU (oracle/_ref_cuda)
    with gpu=True.  Returns (image, seconds of OSEM::reconstruct)."""
    n = len(d1)
    randoms = np.full(n, additive, np.float32)
    oip = ref_image(po, ip)
    return po.ref_osem_listmode(
        ref_scanner(po, sc), oip, sens, d1, d2, tof=tof, randoms=randoms,
        sens_histo=sens_histo, att_params=oip, att_image=mu_np,
        iterations=ITERATIONS, subsets=SUBSETS, tof_fwhm_ps=TOF_FWHM,
        tof_n_std=TOF_NSTD, threads=threads, gpu=gpu)


def our_osem(proj, ip, d1, d2, tof, additive, eff, mu_flat, sens):
    """One reconstruction (ITERATIONS x SUBSETS) of the given device events
    through the public C ABI, as the end-to-end step does: subset-major
    ordering, device corrections, yrtb_osem_listmode."""
    import ctypes
    import pyyrtpet_b200 as yrt
    from pyyrtpet_b200 import _lib as L
    from pyyrtpet_b200.core import _stream
    e = yrt.DeviceEvents(int(d1.numel()), d1, d2, tof=tof)
    e.additive = torch.full((e.count,), additive, device="cuda")
    e, offs = proj.order_events(e, SUBSETS)
    e.sens = proj.gather_crystal_product(eff, e)
    e.att = proj.attenuation_factors(mu_flat, ip, e)
    J = ip.numVoxels
    x = torch.empty(J, device="cuda")
    work = torch.empty(2 * J, device="cuda")
    p = L.yrtb_osem_params(ITERATIONS, SUBSETS, 1.0, 1e-35, 1.19209e-07, 0, 0,
                           None, offs.ctypes.data)
    L.check(L.lib().yrtb_osem_listmode(proj.h, ctypes.byref(e.c()),
                                       sens.data_ptr(), x.data_ptr(),
                                       work.data_ptr(), ctypes.byref(p),
                                       _stream()))
    return x.cpu().numpy().reshape(ip.nz, ip.ny, ip.nx)


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def reference_legs(args, proj, sc, ip, eff, mu, mu_flat, sens, ev_plain,
                   additive, e2e_image):
    """The reference library on this run's workload, with this run's
    sensitivity image (the reference's sensitivity histogram eff1*eff2 is
    filled through its own bin map):
    * cpu_baseline: reference OSEM_CPU (oracle/_ref) on the first
      ref_sample events, timed.  Its image is not compared: with 1M events
      in 10 subsets most voxels of the 10.5M-voxel image get no crossing in
      some subset, and 3 iterations take the whole image to 0, in the
      reference and in this path alike;
    * plain_reference_gpu: reference OSEM_GPU (oracle/_ref_cuda, built for
      sm_100a) on all events, timed (OSEM::reconstruct), and the images of
      the last end-to-end reconstruction (this run's precision) and of a
      mirror-mode reconstruction of the same events against it;
    * the reference GPU sensitivity image against this run's."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    import pyyrtpet_b200 as yrt
    from pyyrtpet_b200 import _lib as L
    threads = os.cpu_count() or 1
    cpu, gpu, par = None, None, {}
    try:
        osc = ref_scanner(po, sc)
        h = po.ref_histo3d_crystal_product(osc, eff.cpu().numpy(), threads)
        sens_np = sens.reshape(ip.nz, ip.ny, ip.nx).cpu().numpy()
        mu_np = mu.cpu().numpy()
        n = min(args.ref_sample, ev_plain.count)
        to_np = lambda t: t.cpu().numpy()
        _, sec = reference_osem(po, sc, ip, to_np(ev_plain.d1[:n]).view(np.uint32),
                                to_np(ev_plain.d2[:n]).view(np.uint32),
                                to_np(ev_plain.tof[:n]), additive, sens_np, h,
                                mu_np, threads, gpu=False)
        cpu = {"value": n * ITERATIONS / sec, "unit": UNIT, "cores": threads,
               "kind": "reference",
               "sample": f"the first {n} of the workload's events, one "
                         f"reconstruction of {ITERATIONS} OSEM iterations x "
                         f"{SUBSETS} subsets (event-iterations/s)"}
        if po.ref_gpu_available() and not args.no_ref_gpu:
            N = ev_plain.count
            img_g, sec_g = reference_osem(
                po, sc, ip, to_np(ev_plain.d1).view(np.uint32),
                to_np(ev_plain.d2).view(np.uint32), to_np(ev_plain.tof),
                additive, sens_np, h, mu_np, threads, gpu=True)
            gpu = {"value": N * ITERATIONS / sec_g, "unit": UNIT,
                   "s_per_reconstruction": sec_g,
                   "what": f"reference OSEM_GPU (YRT-PET compiled for sm_100a "
                           f"from its sources) on the same {N} events, "
                           f"{ITERATIONS} iterations x {SUBSETS} subsets, same "
                           "sensitivity image and corrections; "
                           "OSEM::reconstruct time (its per-subset host "
                           "precompute and copies included), event-iterations/s"}
            par["events"] = N
            if e2e_image is not None:
                par["image_rel_l2_vs_reference_gpu"] = _rel(e2e_image, img_g)
                par["image_precision"] = args.precision
            pp = yrt.ProjectorParams(sc)
            pp.addTOF(TOF_FWHM, TOF_NSTD)
            pp.precision = L.YRTB_MIRROR
            pm = yrt.DeviceProjector(sc, ip, pp)
            mirror = our_osem(pm, ip, ev_plain.d1, ev_plain.d2, ev_plain.tof,
                              additive, eff, mu_flat, sens)
            par["mirror_image_rel_l2_vs_reference_gpu"] = _rel(mirror, img_g)
            if e2e_image is not None:
                par["image_rel_l2_vs_mirror"] = _rel(e2e_image, mirror)
            del pm
            sens_g, _ = po.ref_sensitivity(
                osc, ref_image(po, ip), listmode=True, sens_histo=h,
                att_params=ref_image(po, ip), att_image=mu_np, threads=threads,
                gpu=True)
            par["sensitivity_rel_l2_vs_reference_gpu"] = _rel(sens_np, sens_g[0])
    except Exception as exc:  # reported, never silently replaced
        par["error"] = str(exc)[:300]
        if cpu is None:
            cpu = {"value": None, "unit": UNIT, "cores": threads,
                   "kind": "unavailable", "sample": str(exc)[:200]}
    return cpu, gpu, par


def fp64_parity(sc, ip, proj, ev, n_sample, precision, n_em):
    """This path against the FP64 oracle on the workload's own events:
    forward projections of the first n_sample events (random positive
    image), and one fused EM pass (all corrections) over the first n_em
    events with the initial image.  With the reference's CUDA library built,
    also the reference GPU projector's forward projections of the same sample
    against the same oracle (its own FP32 error)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    import pyyrtpet_b200 as yrt
    threads = os.cpu_count() or 1
    osc = ref_scanner(po, sc)
    oip = ref_image(po, ip)
    lut = po.scanner_lut(osc)
    pr = po.Proj(tof_fwhm_ps=TOF_FWHM, tof_n_std=TOF_NSTD, threads=threads)
    out = {"sample_events": 0, "precision": precision,
           "oracle": "FP64 restatement (oracle/oracle.cpp)"}
    n = min(n_sample, ev.count)
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    img = torch.rand(ip.shape, generator=g, device="cuda") + 0.5
    sub = yrt.DeviceEvents(n, ev.d1[:n], ev.d2[:n], tof=ev.tof[:n])
    got = proj.forward(img, sub).double().cpu().numpy()
    d1 = sub.d1.cpu().numpy().view(np.uint32)
    d2 = sub.d2.cpu().numpy().view(np.uint32)
    tof = sub.tof.cpu().numpy()
    lors, _ = po.lors_from_detpairs(lut, d1, d2)
    img_np = img.cpu().numpy()
    ref = po.project(oip, pr, lors, image=img_np, tof=tof, precision="f64")
    out["fwd_rel_l2"] = _rel(got, ref)
    out["sample_events"] = n
    if po.ref_gpu_available():
        rg = po.ref_project_lm(osc, oip, d1, d2, tof=tof, image=img_np,
                               tof_fwhm_ps=TOF_FWHM, tof_n_std=TOF_NSTD,
                               threads=threads, gpu=True)
        out["reference_gpu_fwd_rel_l2"] = _rel(rg, ref)
    # One EM pass at config scale: the first n_em events (about one subset)
    # with their sensitivity, attenuation and additive terms, image 0.125.
    m = min(n_em, ev.count)
    x = torch.full(ip.shape, 0.125, device="cuda")
    em = torch.zeros(ip.shape, device="cuda")
    sub = yrt.DeviceEvents(m, ev.d1[:m], ev.d2[:m], tof=ev.tof[:m])
    sub.sens, sub.att, sub.additive = ev.sens[:m], ev.att[:m], ev.additive[:m]
    proj.em_step(x, em, sub)
    d1 = sub.d1.cpu().numpy().view(np.uint32)
    d2 = sub.d2.cpu().numpy().view(np.uint32)
    lors, _ = po.lors_from_detpairs(lut, d1, d2)
    ref_em = po.em_step_f64(oip, pr, lors, x.cpu().numpy(),
                            tof=sub.tof.cpu().numpy(),
                            sens=sub.sens.cpu().numpy(), att=sub.att.cpu().numpy(),
                            additive=sub.additive.cpu().numpy())
    out["em_pass_rel_l2"] = _rel(em.cpu().numpy(), ref_em)
    out["em_pass_events"] = m
    return out


def run_reference_arm(args):
    """The reference's own CPU OSEM (YRT-PET compiled from its sources,
    oracle/_ref) on a sample of the workload, on all host threads.  The
    product library is never loaded in this process: the crystal LUT, the
    sensitivity histogram and the sensitivity image come from the reference
    (the image from its OSEM_GPU::generateSensitivityImages when
    oracle/_ref_cuda is built), and the events from the seeded generator
    (torch only), identical to the B200 arm's."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from pyyrtpet_b200 import synthetic as S
    threads = os.cpu_count() or 1
    device = "cuda" if torch.cuda.is_available() else "cpu"
    osc = ref_scanner(po, S.scanner_c2())
    lut = po.ref_scanner_lut(osc)
    sc, ip, ph, eff, evs, mu = build_workload(args.events, device, lut=lut)
    n = min(args.ref_sample, args.events)
    d1 = evs.d1[:n].cpu().numpy().astype(np.uint32)
    d2 = evs.d2[:n].cpu().numpy().astype(np.uint32)
    tof = evs.tof[:n].cpu().numpy().astype(np.float32)
    del evs
    mu_np = mu.cpu().numpy()
    t0 = time.perf_counter()
    h = po.ref_histo3d_crystal_product(osc, eff.cpu().numpy(), threads=threads)
    if po.ref_gpu_available() and torch.cuda.is_available():
        sens, _ = po.ref_sensitivity(osc, ref_image(po, ip), listmode=True,
                                     sens_histo=h, att_params=ref_image(po, ip),
                                     att_image=mu_np, threads=threads, gpu=True)
        sens = sens[0]
        sens_src = ("reference OSEM_GPU::generateSensitivityImages over all "
                    "bins (eff1*eff2 histogram, attenuation)")
    else:
        sens = np.ones((ip.nz, ip.ny, ip.nx), np.float32)
        sens_src = "ones (no reference CUDA library or no GPU here)"
    setup_s = time.perf_counter() - t0
    add = additive_per_event(sc, args.events)
    rates = []
    for i in range(args.warmup + args.steps):
        _, sec = reference_osem(po, sc, ip, d1, d2, tof, add, sens, h, mu_np,
                                threads, gpu=False)
        if i >= args.warmup:
            rates.append(n * ITERATIONS / sec)
    v = float(np.median(rates))
    libs = loaded_libraries()
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * n * ITERATIONS / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded phantom events, C2 shapes)",
            "impl": "reference",
            "config": common_config(world, args.events, n),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads,
                             "kind": "reference",
                             "sample": f"the first {n} of the workload's events, "
                                       f"one reconstruction of {ITERATIONS} OSEM "
                                       f"iterations x {SUBSETS} subsets per step, "
                                       "in event-iterations/s (includes the "
                                       "reference's per-reconstruction "
                                       "correction precompute)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "setup": {"sensitivity_image": sens_src, "setup_s": round(setup_s, 2)},
            "libraries": libs}
    assert not any("libyrtb" in x for x in libs), libs
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ B200 arm -------
def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.config != "c2":
        import bench_configs
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(bench_configs.RUNNERS[args.config](args)), flush=True)
        return
    import ctypes
    import pyyrtpet_b200 as yrt
    from pyyrtpet_b200 import _lib as L
    from pyyrtpet_b200.core import _stream
    from pyyrtpet_b200.distributed import local_subset_range

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    # Rank r holds events [r * n_local, (r + 1) * n_local) of one stream
    # (weak scaling: n_local per GPU); an event's OSEM subset is its global
    # index mod SUBSETS, as the reference's interleaved subsets of the whole
    # stream.
    n_local = args.events
    first_global = rank * n_local
    sc, ip, ph, eff, evs, mu = build_workload(n_local, "cuda",
                                              seed=SEED + 7919 * rank)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(TOF_FWHM, TOF_NSTD)
    pp.precision = (L.YRTB_COMPENSATED if args.precision == "compensated"
                    else L.YRTB_MIRROR)
    pp.deterministic = bool(args.deterministic)
    proj = yrt.DeviceProjector(sc, ip, pp)
    # Correction factors per event, on device: LOR sensitivity eff1*eff2
    # gathered per crystal, ACF via Siddon through the mu-map, flat additive
    # randoms estimate.
    ev = yrt.DeviceEvents.from_arrays(evs.d1.to(torch.int32), evs.d2.to(torch.int32),
                                      tof=evs.tof)
    ev.sens = proj.gather_crystal_product(eff, ev)
    mu_flat = mu.reshape(-1).contiguous()
    ev.att = proj.attenuation_factors(mu_flat, ip, ev)
    additive = additive_per_event(sc, args.events * world)
    ev.additive = torch.full((ev.count,), additive, device="cuda")
    torch.cuda.synchronize()

    # Sensitivity image (setup only, not timed): back projection of all
    # 1.44e9 bins of the scanner's histogram, each with its LOR sensitivity
    # eff1*eff2 and its attenuation factor from the mu-map, in 20
    # phi-interleaved parts, then the reference's hard threshold (1.0).
    sens_pp = yrt.ProjectorParams(sc)
    sens_proj = yrt.DeviceProjector(sc, ip, sens_pp)
    sens = torch.zeros(ip.numVoxels, device="cuda")
    t_sens = time.perf_counter()
    # Each rank back-projects its share of the 20 parts; one all-reduce.
    from pyyrtpet_b200.distributed import sensitivity_histo3d as sharded_sens
    sharded_sens(sens_proj, sens, 20, mu=mu_flat, mu_params=ip, crystal_eff=eff)
    L.check(L.lib().yrtb_apply_threshold(sens.data_ptr(), sens.data_ptr(),
                                         ip.numVoxels, 1, 1, 1.0, 0.0, 0.0,
                                         1.0, 0.0, _stream()))
    torch.cuda.synchronize()
    sens_setup_s = time.perf_counter() - t_sens
    sens_sub = (sens / SUBSETS).contiguous()
    J = ip.numVoxels
    img = torch.full((J,), 0.125, device="cuda")
    img.mul_((sens > 0).float())
    em = torch.zeros(J, device="cuda")
    # Image layout of the timed EM passes (set-up: the image and the subset
    # sensitivity converted once; the EM update is elementwise).
    tiled = args.layout == "tile" and not args.deterministic
    if tiled:
        proj.set_image_layout(L.YRTB_LAYOUT_TILE_4X2)
        img = proj.to_layout(img, ip, L.YRTB_LAYOUT_TILE_4X2)
        sens_sub = proj.to_layout(sens_sub, ip, L.YRTB_LAYOUT_TILE_4X2)

    # Launch configuration: timed on a sample of subset 0 (setup, not timed;
    # a calibration done once per projector, like a library's algorithm
    # search), then used by the ordered and end-to-end forms.
    tune = None
    if not args.no_autotune:
        tune = proj.autotune(img, ev, SUBSETS)
        if args.tune_report and rank == 0:
            with open(args.tune_report, "w") as f:
                json.dump(tune, f, indent=1)
    if args.vector_groups >= 0:
        proj.set_launch(**dict(proj.get_launch(), vector_groups=args.vector_groups))
    launch = proj.get_launch()

    # Plain form: events in file order, subset = interleaved stride (the
    # reference's batching).  Ordered form: subset-major, LOR-sorted copy.
    ev_plain = ev
    ev, offsets = proj.order_events(ev_plain, SUBSETS,
                                    first_global_index=first_global)
    torch.cuda.synchronize()

    # Algorithmic traffic of the fused EM kernel: per event 24 B of event data
    # (d1, d2, tof, sens, att, additive) + 4 B per crossing for the forward
    # gather + 8 B per crossing for the back-projection read-modify-write.
    counts = proj.count_crossings(ev)
    n_vox_total = float(counts.double().sum().item())
    alg_bytes_iter = 24.0 * ev.count + 12.0 * n_vox_total
    del counts

    st = torch.cuda.current_stream()
    s_ptr = _stream()
    lib = L.lib()
    evc = ev.c()
    launches = [0]

    evc_plain = ev_plain.c()

    def step(record=None, plain=False):
        for s in range(SUBSETS):
            L.check(lib.yrtb_fill(em.data_ptr(), J, 0.0, s_ptr))
            if plain:
                r = L.yrtb_range(*local_subset_range(ev_plain.count, first_global,
                                                     SUBSETS, s))
            else:
                r = L.yrtb_range(int(offsets[s]), 1,
                                 int(offsets[s + 1] - offsets[s]))
            if record is not None:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
            L.check(lib.yrtb_em_step(proj.h, img.data_ptr(), em.data_ptr(),
                                     ctypes.byref(evc_plain if plain else evc),
                                     r, 1.0, 1e-35, s_ptr))
            if record is not None:
                b.record(st)
                record.append((a, b))
            if dist is not None:
                dist.all_reduce(em)
            L.check(lib.yrtb_em_update(img.data_ptr(), em.data_ptr(),
                                       sens_sub.data_ptr(), J, 1, 1, 1.19209e-07,
                                       None, s_ptr))
            launches[0] += 3

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clk_path = os.path.join(tempfile.mkdtemp(prefix="yrtb_clocks_"), f"clocks_rank{rank}.csv")
    sampler = clocks_sampler(clk_path) if rank == 0 else None
    time.sleep(0.5)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches[0] = 0
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    em_events = []
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select these launches
    t0.record(st)
    for _ in range(args.steps):
        step(record=em_events)
    t1.record(st)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    if dist is not None:
        dist.barrier()
    if sampler is not None:
        time.sleep(0.3)
        sampler.terminate()
    ms = t0.elapsed_time(t1) / args.steps
    em_ms = float(np.mean([a.elapsed_time(b) for a, b in em_events]))
    if dist is not None:
        tt = torch.tensor([ms, em_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, em_ms = tt.tolist()
    total_events = ev.count * world
    value = total_events / (ms * 1e-3)
    timed_launches = launches[0]

    # Plain (file-order) form on the same GPU, for the batched-vs-plain ratio,
    # with the reference's launch shape (one thread per event, 256-thread
    # blocks) and image layout (row-major).
    if tiled:
        img = proj.to_layout(img, ip, L.YRTB_LAYOUT_ROW_MAJOR)
        sens_sub = proj.to_layout(sens_sub, ip, L.YRTB_LAYOUT_ROW_MAJOR)
        proj.set_image_layout(L.YRTB_LAYOUT_ROW_MAJOR)
    proj.set_launch(256, 1, launch["bucket_shift"], launch["order"],
                    launch["tile_shift"], 0)
    for _ in range(1):
        step(plain=True)
    pa = torch.cuda.Event(enable_timing=True)
    pb = torch.cuda.Event(enable_timing=True)
    pa.record(st)
    for _ in range(args.steps):
        step(plain=True)
    pb.record(st)
    torch.cuda.synchronize()
    plain_ms = pa.elapsed_time(pb) / args.steps
    if dist is not None:
        tt = torch.tensor([plain_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        plain_ms = tt.item()
    proj.set_launch(**launch)

    # ---- e2e: public OSEM API from pinned host buffers (one reconstruction
    # per step).  The events of step k+1 are copied on a second stream while
    # step k computes (two device buffers); every step's copy is still inside
    # the timed region.
    e2e = None
    e2e_image = None
    if not args.no_e2e:
        h_d1 = evs.d1.to(torch.int32).cpu().pin_memory()
        h_d2 = evs.d2.to(torch.int32).cpu().pin_memory()
        h_tof = evs.tof.cpu().pin_memory()
        h_add = ev_plain.additive.cpu().pin_memory()
        host = (h_d1, h_d2, h_tof, h_add)
        bufs = [tuple(torch.empty_like(h, device="cuda") for h in host)
                for _ in range(2)]
        h_img = torch.empty(J, dtype=torch.float32).pin_memory()
        eff_d = eff
        copy_stream = torch.cuda.Stream()
        copied = [torch.cuda.Event(), torch.cuda.Event()]
        released = [torch.cuda.Event(), torch.cuda.Event()]
        for r in released:
            r.record(st)

        def upload(k):
            b = bufs[k % 2]
            copy_stream.wait_event(released[k % 2])  # its previous step is done
            with torch.cuda.stream(copy_stream):
                for dst, src in zip(b, host):
                    dst.copy_(src, non_blocking=True)
            copied[k % 2].record(copy_stream)

        def e2e_step(k, last):
            st.wait_event(copied[k % 2])
            if not last:
                upload(k + 1)
            d_d1, d_d2, d_tof, d_add = bufs[k % 2]
            e = yrt.DeviceEvents(int(d_d1.numel()), d_d1, d_d2, tof=d_tof)
            e.additive = d_add
            # Subset-major order first, then the corrections on the ordered
            # arrays (the attenuation walks run on grouped rays).
            e, offs = proj.order_events(e, SUBSETS, first_global_index=first_global)
            released[k % 2].record(st)  # the ordered copy no longer reads it
            e.sens = proj.gather_crystal_product(eff_d, e)
            e.att = proj.attenuation_factors(mu_flat, ip, e)
            x = torch.full((J,), 0.125, device="cuda")
            if dist is None:
                work = torch.empty(2 * J, device="cuda")
                p = L.yrtb_osem_params(ITERATIONS, SUBSETS, 1.0, 1e-35, 1.19209e-07,
                                       0, 0, None, offs.ctypes.data)
                L.check(lib.yrtb_osem_listmode(proj.h, ctypes.byref(e.c()),
                                               sens.data_ptr(), x.data_ptr(),
                                               work.data_ptr(), ctypes.byref(p),
                                               s_ptr))
            else:
                # Sharded reconstruction: the EM image is summed over ranks
                # once per subset (NCCL) between the EM pass and the update.
                from pyyrtpet_b200.distributed import osem_listmode
                osem_listmode(proj, e, offs, sens, x, ITERATIONS, SUBSETS,
                              first_global_index=first_global)
            h_img.copy_(x, non_blocking=True)

        def run_steps(n, a=None):
            if a is not None:
                copy_stream.wait_event(a)
            upload(0)
            for k in range(n):
                e2e_step(k, k == n - 1)

        run_steps(max(1, args.warmup))
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("e2e")  # lets a profiler select these launches
        a.record(st)
        run_steps(args.steps, a)
        b.record(st)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        e2e_ms = a.elapsed_time(b) / args.steps
        if dist is not None:
            tt = torch.tensor([e2e_ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_ms = tt.item()
        e2e_image = h_img.numpy().reshape(ip.nz, ip.ny, ip.nx).copy()
        e2e = {"value": total_events * ITERATIONS / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(sum(h.numel() * h.element_size() for h in host)),
               "d2h_bytes_per_step": int(J * 4), "ms_per_step": e2e_ms,
               "iterations_per_step": ITERATIONS,
               "path": ("yrtb_osem_listmode (C ABI)" if dist is None else
                        "pyyrtpet_b200.distributed.osem_listmode (C ABI EM "
                        "passes, NCCL all-reduce per subset)") + " from pinned host events; "
                       "per step: H2D events (detector pairs, TOF, randoms "
                       "estimate; double-buffered: the next step's copy "
                       "overlaps this step's compute), event ordering, device "
                       "corrections (eff1*eff2 gather, attenuation walks), one "
                       "reconstruction of 3 OSEM iterations x 10 subsets, D2H "
                       "image"}

    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes_iter / SUBSETS / (em_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": None,
                "kernel": "k_events<OP_EM, K_SIDDON, TOF> (fused fwd->ratio->bwd)",
                "alg_bytes_per_launch": alg_bytes_iter / SUBSETS,
                "mean_crossings_per_event": n_vox_total / ev.count,
                "em_kernel_ms_per_launch": em_ms}
    prof = os.path.join(ROOT, "profiles", "em_siddon_tof_c2_traffic.json")
    if os.path.exists(prof):
        try:
            roofline["traffic"] = json.load(open(prof))["dram_bytes_per_launch"]
        except Exception:
            pass
    # The kernel's L2 ceiling: its L2 requests per event (reads of the image
    # by the forward walk, float4 reductions by the back projection; ncu
    # counts for the same launch configuration) at the measured L2 request
    # rate of the same mix on this GPU.
    l2prof = os.path.join(ROOT, "profiles", "em_siddon_tof_c2_l2.json")
    if not args.no_l2_peak and os.path.exists(l2prof):
        rates = measured_l2_request_rates(J)
        l2 = {"peak_requests_per_s": rates,
              "peak_source": "measured live (libyrtb_l2bench.so: random aligned groups "
                             "in an L2-resident buffer of the image's size)"}
        # ncu request counts per event, one entry per launch configuration
        # they were taken with; the first entry that matches this run's.
        entries = json.load(open(l2prof))["entries"]
        launch = dict(proj.get_launch(), image_layout=(L.YRTB_LAYOUT_TILE_4X2 if tiled
                                                       else L.YRTB_LAYOUT_ROW_MAJOR))
        cnt = next((c for c in entries
                    if all(launch.get(k) == v for k, v in c["launch"].items())), None)
        if cnt is not None:
            reqs = (cnt["red_requests_per_event"] + cnt["read_requests_per_event"]) \
                * ev.count / SUBSETS
            l2["requests_per_launch"] = reqs
            l2["requests_source"] = cnt["source"]
            l2["achieved_requests_per_s"] = reqs / (em_ms * 1e-3)
            # The ceiling of a 1:1 mix of reads and reductions: the faster of
            # the two ways of mixing them.
            mix = max(rates[L2_MODES[3]], rates[L2_MODES[4]])
            l2["peak_mix_requests_per_s"] = mix
            roofline["l2_frac"] = l2["achieved_requests_per_s"] / mix
        else:
            l2["requests_per_launch"] = None
            l2["requests_source"] = ("ncu counts were taken with launches "
                                     f"{[c['launch'] for c in entries]}, this run "
                                     f"chose {launch}")
        roofline["l2"] = l2

    cpu = None
    parity = None
    plain_ref_gpu = None
    par_ref = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # Parity and baseline legs (not timed): forward projections of a
        # sample against the FP64 oracle; then the reference library itself
        # on the same events with the same sensitivity image and corrections.
        try:
            parity = fp64_parity(sc, ip, proj, ev_plain, args.parity_sample,
                                 args.precision, ev_plain.count // SUBSETS)
        except Exception as exc:
            parity = {"error": str(exc)[:200]}
        cpu, plain_ref_gpu, par_ref = reference_legs(
            args, proj, sc, ip, eff, mu, mu_flat, sens, ev_plain, additive,
            e2e_image)

    if rank == 0:
        clocks = summarize_clocks(clk_path, local) if sampler else None
        line = {"metric": METRIC, "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded phantom events, C2 shapes)",
                "config": common_config(world, args.events,
                                        min(args.ref_sample, args.events)),
                "mode": {"precision": args.precision,
                         "deterministic": bool(args.deterministic),
                         "image_layout": "tile_4x2" if tiled else "row_major",
                         "launch": launch,
                         "autotune": None if tune is None else {
                             "sample_events": tune["sample_events"],
                             "candidates": len(tune["tried"]),
                             "best_ms": min(ms for _, ms in tune["tried"]) if tune["tried"] else None,
                             "default_ms": next((ms for c, ms in tune["tried"]
                                                 if c == {"block": 256, "threads_per_lor": 1,
                                                          "bucket_shift": 3, "order": 0,
                                                          "tile_shift": 1,
                                                          "vector_groups": 2}), None)},
                         "sensitivity_setup_s": round(sens_setup_s, 3)},
                "gpu_launches": timed_launches,
                "plain": {"value": total_events / (plain_ms * 1e-3),
                          "ms_per_step": plain_ms,
                          "what": "same kernels, events in file order with "
                                  "interleaved subsets (the reference's "
                                  "single-frame batching)"},
                "osem_s_per_iteration": ms * 1e-3,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "plain_reference_gpu": plain_ref_gpu,
                "batched_vs_plain_reference_gpu": (
                    e2e["value"] / plain_ref_gpu["value"]
                    if e2e and plain_ref_gpu and plain_ref_gpu.get("value") else None),
                "parity_vs_fp64": parity,
                "parity_vs_reference": par_ref,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
