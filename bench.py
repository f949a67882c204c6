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
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c2mr", "c3", "c4", "c5", "psf", "lrem"],
                    help="c2 (default) is the headline workload; the others "
                         "run bench_configs.py")
    ap.add_argument("--cfg-events", type=int, default=0,
                    help="override the event count of --config c1/c2mr/c3/c4/c5")
    return ap.parse_args()


# ----------------------------------------------------------------- workload --
def build_workload(n_events, device, seed=SEED):
    from pyyrtpet_b200 import synthetic as S
    import pyyrtpet_b200 as yrt
    sc = S.scanner_c2()
    ip = S.image_c2()
    ph = S.Phantom(cyl_half_length=sc.axialFOV / 2)
    eff = S.crystal_efficiencies(sc, seed + 1, device=device)
    ev = S.generate_events(sc, n_events, seed, phantom=ph, tof_fwhm_ps=TOF_FWHM,
                           mu_per_mm=0.0096, crystal_eff=eff,
                           randoms_fraction=0.2, device=device)
    mu = ph.mu_image(ip, device=device)
    return sc, ip, ph, eff, ev, mu


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


# --------------------------------------------------------- reference (CPU) --
def reference_rate(sc, ip, ev, mu, eff_np, n_sample, threads, iterations=1):
    """Reference YRT-PET CPU OSEM (oracle/_ref) on a bounded sample of the
    same workload; returns (events/s, kind, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    e = {"d1": ev.d1[:n_sample].cpu().numpy().astype(np.uint32),
         "d2": ev.d2[:n_sample].cpu().numpy().astype(np.uint32),
         "tof": ev.tof[:n_sample].cpu().numpy().astype(np.float32)}
    n = len(e["d1"])
    osc = po.Scanner(sc.axialFOV, sc.crystalSize_z, sc.crystalSize_trans,
                     sc.crystalDepth, sc.scannerRadius, sc.detsPerRing,
                     sc.numRings, sc.numDOI, sc.maxRingDiff, sc.minAngDiff,
                     sc.detsPerBlock)
    oip = po.ImageParams(ip.nx, ip.ny, ip.nz, ip.length_x, ip.length_y, ip.length_z)
    sens = np.ones((ip.nz, ip.ny, ip.nx), np.float32)
    randoms = np.full(n, 1e-3, np.float32)
    if po.ref_available():
        _, sec = po.ref_osem_listmode(
            osc, oip, sens, e["d1"], e["d2"], tof=e["tof"], randoms=randoms,
            att_params=oip, att_image=mu.cpu().numpy(), iterations=iterations,
            subsets=SUBSETS, tof_fwhm_ps=TOF_FWHM, tof_n_std=TOF_NSTD,
            threads=threads)
        return n * iterations / sec, "reference", sec
    # Fallback: the oracle's FP64 EM pass (a port, not the reference).
    lut = po.scanner_lut(osc)
    lors, _ = po.lors_from_detpairs(lut, e["d1"], e["d2"])
    img = np.full((1, ip.nz, ip.ny, ip.nx), 0.125, np.float32)
    t0 = time.perf_counter()
    for s in range(SUBSETS):
        sl = slice(s, n, SUBSETS)
        po.em_step_f64(po.ImageParams(ip.nx, ip.ny, ip.nz, ip.length_x,
                                      ip.length_y, ip.length_z),
                       po.Proj(tof_fwhm_ps=TOF_FWHM, tof_n_std=TOF_NSTD,
                               threads=threads),
                       lors[sl], img, tof=e["tof"][sl], additive=randoms[sl])
    sec = time.perf_counter() - t0
    return n / sec, "port", sec


def fp64_parity(sc, ip, proj, ev, n_sample, precision):
    """rel-L2 of this path's forward projections vs the FP64 oracle on the
    first n_sample events (non-zero random image)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    import pyyrtpet_b200 as yrt
    n = min(n_sample, ev.count)
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    img = torch.rand(ip.shape, generator=g, device="cuda") + 0.5
    sub = yrt.DeviceEvents(n, ev.d1[:n], ev.d2[:n], tof=ev.tof[:n])
    got = proj.forward(img, sub).double().cpu().numpy()
    osc = po.Scanner(sc.axialFOV, sc.crystalSize_z, sc.crystalSize_trans,
                     sc.crystalDepth, sc.scannerRadius, sc.detsPerRing,
                     sc.numRings, sc.numDOI, sc.maxRingDiff, sc.minAngDiff,
                     sc.detsPerBlock)
    lut = po.scanner_lut(osc)
    d1 = sub.d1.cpu().numpy().view(np.uint32)
    d2 = sub.d2.cpu().numpy().view(np.uint32)
    lors, _ = po.lors_from_detpairs(lut, d1, d2)
    oip = po.ImageParams(ip.nx, ip.ny, ip.nz, ip.length_x, ip.length_y,
                         ip.length_z)
    ref = po.project(oip, po.Proj(tof_fwhm_ps=TOF_FWHM, tof_n_std=TOF_NSTD,
                                  threads=os.cpu_count() or 1),
                     lors, image=img.cpu().numpy(), tof=sub.tof.cpu().numpy(),
                     precision="f64")
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return {"fwd_rel_l2": err, "sample_events": n, "precision": precision,
            "oracle": "FP64 restatement (oracle/oracle.cpp)"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sc, ip, ph, eff, ev, mu = build_workload(max(args.ref_sample, 1000), "cpu")
    rates = []
    for i in range(args.warmup + args.steps):
        r, kind, sec = reference_rate(sc, ip, ev, mu, None, args.ref_sample,
                                      threads, ITERATIONS)
        if i >= args.warmup:
            rates.append(r)
    v = float(np.median(rates))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * args.ref_sample * ITERATIONS / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded phantom events, C2 shapes)",
            "impl": "reference",
            "config": {"workload": WORKLOAD,
                       "sample_events": args.ref_sample, "subsets": SUBSETS},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads,
                             "kind": kind,
                             "sample": f"{args.ref_sample} events of the workload, "
                                       f"one reconstruction of {ITERATIONS} OSEM "
                                       f"iterations x {SUBSETS} subsets, in "
                                       "event-iterations/s (includes the "
                                       "reference's per-reconstruction "
                                       "correction precompute)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
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

    n_local = args.events
    sc, ip, ph, eff, evs, mu = build_workload(n_local, "cuda",
                                              seed=SEED + 7919 * rank)
    pp = yrt.ProjectorParams(sc)
    pp.addTOF(TOF_FWHM, TOF_NSTD)
    pp.precision = (L.YRTB_COMPENSATED if args.precision == "compensated"
                    else L.YRTB_MIRROR)
    pp.deterministic = bool(args.deterministic)
    proj = yrt.DeviceProjector(sc, ip, pp)
    # Correction factors per event, on device (sens = eff1*eff2 histogram
    # gather is equivalent to the direct product here; ACF via Siddon
    # through the mu-map; flat additive randoms estimate).
    ev = yrt.DeviceEvents.from_arrays(evs.d1.to(torch.int32), evs.d2.to(torch.int32),
                                      tof=evs.tof)
    ev.sens = (eff[evs.d1] * eff[evs.d2]).float().contiguous()
    mu_flat = mu.reshape(-1).contiguous()
    ev.att = proj.attenuation_factors(mu_flat, ip, ev)
    n_rand_lors = float(sc.getNumDets()) ** 2 / 2 * 0.45
    ev.additive = torch.full((ev.count,), 0.2 * ev.count / n_rand_lors,
                             device="cuda")
    torch.cuda.synchronize()

    # Sensitivity image (setup only, not timed): back projection of all
    # 1.44e9 bins of the scanner's histogram, with the attenuation factor of
    # each bin from the mu-map, in 20 phi-interleaved parts.
    sens_pp = yrt.ProjectorParams(sc)
    sens_proj = yrt.DeviceProjector(sc, ip, sens_pp)
    sens = torch.zeros(ip.numVoxels, device="cuda")
    t_sens = time.perf_counter()
    for part in range(20):
        sens_proj.sensitivity_histo3d(sens, 20, part, mu=mu_flat, mu_params=ip)
    torch.cuda.synchronize()
    sens_setup_s = time.perf_counter() - t_sens
    sens_sub = (sens / SUBSETS).contiguous()
    J = ip.numVoxels
    img = torch.full((J,), 0.125, device="cuda")
    img.mul_((sens > 0).float())
    em = torch.zeros(J, device="cuda")

    # Launch configuration: timed on a sample of subset 0 (setup, not timed;
    # a calibration done once per projector, like a library's algorithm
    # search), then used by the ordered and end-to-end forms.
    tune = None
    if not args.no_autotune:
        tune = proj.autotune(img, ev, SUBSETS)
        if args.tune_report and rank == 0:
            with open(args.tune_report, "w") as f:
                json.dump(tune, f, indent=1)
    launch = proj.get_launch()

    # Plain form: events in file order, subset = interleaved stride (the
    # reference's batching).  Ordered form: subset-major, LOR-sorted copy.
    ev_plain = ev
    ev, offsets = proj.order_events(ev_plain, SUBSETS)
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
                r = L.yrtb_range(s, SUBSETS, 0)
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
    # blocks).
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
    if not args.no_e2e:
        h_d1 = evs.d1.to(torch.int32).cpu().pin_memory()
        h_d2 = evs.d2.to(torch.int32).cpu().pin_memory()
        h_tof = evs.tof.cpu().pin_memory()
        bufs = [tuple(torch.empty_like(h, device="cuda") for h in (h_d1, h_d2, h_tof))
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
                for dst, src in zip(b, (h_d1, h_d2, h_tof)):
                    dst.copy_(src, non_blocking=True)
            copied[k % 2].record(copy_stream)

        def e2e_step(k, last):
            st.wait_event(copied[k % 2])
            if not last:
                upload(k + 1)
            d_d1, d_d2, d_tof = bufs[k % 2]
            e = yrt.DeviceEvents(int(d_d1.numel()), d_d1, d_d2, tof=d_tof)
            e.additive = ev_plain.additive
            # Subset-major order first, then the corrections on the ordered
            # arrays (the attenuation walks run on grouped rays).
            e, offs = proj.order_events(e, SUBSETS)
            released[k % 2].record(st)  # the ordered copy no longer reads it
            e.sens = (eff_d[e.d1.long()] * eff_d[e.d2.long()]).contiguous()
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
                osem_listmode(proj, e, offs, sens, x, ITERATIONS, SUBSETS)
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
        a.record(st)
        run_steps(args.steps, a)
        b.record(st)
        torch.cuda.synchronize()
        e2e_ms = a.elapsed_time(b) / args.steps
        if dist is not None:
            tt = torch.tensor([e2e_ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_ms = tt.item()
        e2e = {"value": total_events * ITERATIONS / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(h_d1.numel() * 12),
               "d2h_bytes_per_step": int(J * 4), "ms_per_step": e2e_ms,
               "iterations_per_step": ITERATIONS,
               "path": ("yrtb_osem_listmode (C ABI)" if dist is None else
                        "pyyrtpet_b200.distributed.osem_listmode (C ABI EM "
                        "passes, NCCL all-reduce per subset)") + " from pinned host events; "
                       "per step: H2D events (double-buffered: the next "
                       "step's copy overlaps this step's compute), event "
                       "ordering, device corrections, one reconstruction of 3 "
                       "OSEM iterations x 10 subsets, D2H image"}

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

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # CPU leg: forward projections of a sample of the workload's events in
        # this run's precision mode against the FP64 oracle.
        try:
            parity = fp64_parity(sc, ip, proj, ev_plain, args.parity_sample,
                                 args.precision)
        except Exception as exc:
            parity = {"error": str(exc)[:200]}
        try:
            r, kind, sec = reference_rate(sc, ip, evs, mu, None,
                                          min(args.ref_sample, ev.count),
                                          os.cpu_count() or 1, ITERATIONS)
            cpu = {"value": r, "unit": UNIT, "cores": os.cpu_count(),
                   "kind": kind,
                   "sample": f"{min(args.ref_sample, ev.count)} events of this "
                             f"workload, one reconstruction of {ITERATIONS} OSEM "
                             f"iterations x {SUBSETS} subsets (event-iterations/s)"}
        except Exception as exc:  # reported, never silently replaced
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                   "kind": "unavailable", "sample": str(exc)[:200]}

    if rank == 0:
        clocks = summarize_clocks(clk_path, local) if sampler else None
        line = {"metric": METRIC, "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded phantom events, C2 shapes)",
                "config": {"workload": WORKLOAD,
                           "events_per_gpu": ev.count, "subsets": SUBSETS,
                           "precision": args.precision,
                           "deterministic": bool(args.deterministic),
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
                           "sensitivity": {"bins": "all 1.44e9 histogram bins, "
                                                   "attenuation from the mu-map",
                                           "setup_s": round(sens_setup_s, 3)},
                           "l2": "event arrays (1.2 GB) larger than L2; "
                                 "image (42 MB) L2-resident by design",
                           "parallelism": f"dp{world} (events sharded, EM image "
                                          "all-reduced per subset)"},
                "gpu_launches": timed_launches,
                "plain": {"value": total_events / (plain_ms * 1e-3),
                          "ms_per_step": plain_ms,
                          "what": "same kernels, events in file order with "
                                  "interleaved subsets (the reference's "
                                  "single-frame batching)"},
                "osem_s_per_iteration": ms * 1e-3,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "parity_vs_fp64": parity,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
