#!/usr/bin/env python
"""Projector throughput benchmark (one JSON line on rank 0).

Default workload ``cbct``: cone-beam CT with a 512 x 512 flat panel (0.4 mm
pixels), 360 projections over 360 degrees, source-origin 500 mm and
source-detector 1000 mm, a 256^3 volume of 0.25 mm voxels, a seeded 3-D
ellipsoid (Shepp-Logan-style) phantom with attenuation 0-0.02 /mm, Poisson
transmission data at I0 = 1e5 linearised as log(I0 / I), branchless
distance-driven projector (type 5), PDHG with a TV-gradient term.
One step = one PDHG iteration over all 360 projections: forward projection
(94,371,840 rays), dual update, backprojection, TV gradient and primal update.

metric: rays/s of FP+BP pairs (rays forward- and back-projected per second).
``value`` times device-resident data with CUDA events; ``e2e`` times a
forward+back projection through the C-ABI with the image copied in from
pinned host memory and the backprojection copied out, every step.
``cpu_baseline``: the reference has no CPU code for projector type 5
(proj.py:1212-1213 rejects it), so the CPU figure is the FP64 OpenMP
restatement of its kernels on a bounded sample, labelled "port".

Workload ``dynpet``: 24-frame dynamic PET on a 384-crystal x 32-ring
scanner, 256 x 192 x 63 sinograms, 128 x 128 x 63 image, improved Siddon;
one step = forward projection of all frames then backprojection of all
frames; CPU baseline = the reference's own OpenMP projector.

--impl reference times the reference CPU implementation of the same step
(the OpenMP projector for dynpet, the restatement for cbct) with all host
threads on a bounded sample.  Under torchrun only rank 0 runs it.
Multi-GPU: replicas (each rank runs its own copy of the workload, no
collective on the data path); value = all ranks' rays / max rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes (read + write) per launch from ncu captures, scaled to the full
# workload by rays where the capture was smaller; see profiles/ for the
# captures they come from.
PROFILED_TRAFFIC = {
    # DRAM bytes read + written per launch, from the ncu captures summarised
    # in profiles/: bdd_cbct_capture.md (36-view capture x 10) and
    # siddon_dynpet_launches.md (full-size capture)
    ("cbct", "bdd_fp"): 9.46e9,
    ("cbct", "bdd_bp"): 3.76e8,
    ("dynpet", "siddon_fp"): 3.81e8,
    ("dynpet", "siddon_bp"): 6.59e9,   # 3 launches of k_sm_bp_sl (8 frames each) per call
    # interp_tof_capture.md: one subset's forward launch (16 per step)
    ("interp_tof", "interp_fp"): 5.60e6,
}
# What bounds each kernel instead of HBM (the volumes and images are
# L2-resident, so DRAM moves a few per cent of the cache-less bytes): the
# issue-active and SM-throughput percentages of the same ncu captures.
PROFILED_LIMITER = {
    ("cbct", "bdd_fp"): {"issue_active_pct": 80.4, "sm_throughput_pct": 75.5, "dram_pct": 7.6},
    ("cbct", "bdd_bp"): {"issue_active_pct": 72.9, "sm_throughput_pct": 71.8, "dram_pct": 0.35},
    ("dynpet", "siddon_fp"): {"issue_active_pct": 66.5, "l1tex_pct": 92.0, "dram_pct": 1.0},
    ("dynpet", "siddon_bp"): {"issue_active_pct": 10.7, "l1tex_pct": 94.0, "dram_pct": 21.8},
    ("interp_tof", "interp_fp"): {"issue_active_pct": 84.9, "sm_throughput_pct": 78.6, "dram_pct": 0.01},
}
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="cbct",
                   choices=["cbct", "cbct_small", "dynpet", "dynpet_small", "fanbeam64", "fanbeam64_small",
                            "interp_tof", "interp_tof_small", "tube", "tube_small"])
    p.add_argument("--frames", type=int, default=None)
    p.add_argument("--views", type=int, default=None,
                   help="cbct: number of projections (fewer than 360 only for short profiling captures)")
    p.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-learned", action="store_true", help="skip the learned-vs-plain OSEM time-to-logL leg")
    p.add_argument("--no-legs", action="store_true",
                   help="skip the Siddon dynamic-PET and type-4 TOF legs of the default line")
    p.add_argument("--tuning", default=None,
                   help="fixed launch shapes instead of the autotuner, e.g. bdd_fp_columns=16,bdd_bp_zrun=8")
    return p.parse_args()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def dynamic_pet_options(small=False):
    from omega_b200.projector import geometry as geo
    from omega_b200.projector import proj
    o = proj.projectorClass()
    rings = 8 if small else 32
    o.blocks_per_ring, o.cryst_per_block = 16, 24
    o.cryst_per_block_axial, o.linear_multip = rings, 1
    o.rings = rings
    o.det_per_ring = o.det_w_pseudo = 384
    o.diameter = 600.
    o.cr_p = math.pi * 600. / 384.
    o.cr_pz = 4.0
    o.FOVa_x = o.FOVa_y = 300.
    o.Nx = o.Ny = 128
    o.Nz = 2 * rings - 1
    o.axial_fov = 2.0 * o.Nz
    o.span, o.ring_difference = 3, rings - 1
    o.Ndist, o.Nang = 256, 192
    o.NSinos = 2 * rings - 1
    o.TotSinos = int(np.sum(geo.default_segment_table(rings, 3, rings - 1, 2 * rings - 1)))
    o.projector_type = 1
    o.subsets, o.subsetType = 16, 8
    o.verbose = 0
    o.addProjector()
    return o


def dynamic_images(o, frames, seed=2024):
    """Seeded phantom: warm cylinder with four hot and one cold sphere, each
    region scaled per frame by a gamma-variate time-activity curve."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = int(o.Nx[0]), int(o.Ny[0]), int(o.Nz[0])
    dx, dz = float(o.dx[0]), float(o.dz[0])
    xs = (np.arange(nx) + 0.5) * dx + float(o.bx[0])
    zs = (np.arange(nz) + 0.5) * dz + float(o.bz[0])
    X, Y, Z = np.meshgrid(xs, xs, zs, indexing="ij")
    regions = [((X ** 2 + Y ** 2) < 120. ** 2).astype(np.float32)]
    for _ in range(5):
        c = rng.uniform(-60, 60, 3) * np.array([1, 1, 0.3])
        r = rng.uniform(10, 25)
        regions.append((((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) < r * r).astype(np.float32))
    t = np.linspace(0.5, 60., frames)
    imgs = np.zeros((frames, nx * ny * nz), dtype=np.float32)
    for k, reg in enumerate(regions):
        a, b = rng.uniform(1.5, 3.5), rng.uniform(2., 10.)
        tac = (t / b) ** a * np.exp(-(t - b) / b) + 0.1
        flat = reg.ravel(order="F")
        imgs += np.outer(tac, flat).astype(np.float32)
    return imgs


def tof_pet_options(small=False, **extra):
    """The precision workload: 672 crystals x 55 rings (42 blocks of 16, ring
    diameter 856 mm), 400 radial x 336 angles x 109 span-3 sinograms with 15
    TOF bins of 200 ps FWHM covering +-424 mm (the FOV diagonal), a
    200 x 200 x 109 image over 600 x 600 x 436 mm, projector type 4, 16
    subsets.  ``small``: 11 rings, 22 sinograms, 100 x 100 x 21 image."""
    from omega_b200.projector import geometry as geo
    from omega_b200.projector import proj
    c = 2.99792458e11  # mm/s
    rings, nz, nx = (11, 21, 100) if small else (55, 109, 200)
    o = proj.projectorClass()
    o.blocks_per_ring, o.cryst_per_block, o.cryst_per_block_axial, o.linear_multip = 42, 16, rings, 1
    o.rings = rings
    o.det_per_ring = o.det_w_pseudo = 672
    o.diameter = 856.
    o.cr_p = math.pi * 856. / 672.
    o.cr_pz = 4.0
    o.FOVa_x = o.FOVa_y = 600.
    o.axial_fov = 436. * nz / 109.
    o.Nx = o.Ny = nx
    o.Nz = nz
    o.span, o.ring_difference = 3, rings - 1
    o.Ndist, o.Nang = (400, 336) if not small else (200, 168)
    o.NSinos = nz
    o.TotSinos = int(np.sum(geo.default_segment_table(rings, 3, rings - 1, nz)))
    o.TOF_bins = o.TOF_bins_used = 15
    o.TOF_FWHM = 200e-12
    o.TOF_width = 848.0 / 15 / (c / 2)
    o.projector_type = 4
    o.subsets, o.subsetType = 16, 8
    o.verbose = 0
    for k, v in extra.items():
        setattr(o, k, v)
    o.addProjector()
    return o


def tof_phantom(o, seed=7):
    """Seeded anthropomorphic-style ellipsoid phantom: elliptic body, two
    lung-like cold ellipsoids, a warm organ and hot lesions."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = int(o.Nx[0]), int(o.Ny[0]), int(o.Nz[0])
    xs = (np.arange(nx) + 0.5) * float(o.dx[0]) + float(o.bx[0])
    ys = (np.arange(ny) + 0.5) * float(o.dy[0]) + float(o.by[0])
    zs = (np.arange(nz) + 0.5) * float(o.dz[0]) + float(o.bz[0])
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    img = 1.0 * ((X / 220.) ** 2 + (Y / 150.) ** 2 < 1)
    for sx in (-90., 90.):
        img[((X - sx) / 60.) ** 2 + (Y / 80.) ** 2 + (Z / 150.) ** 2 < 1] = 0.3
    img[((X - 30.) / 70.) ** 2 + ((Y + 40.) / 50.) ** 2 + ((Z + 60.) / 80.) ** 2 < 1] = 2.0
    for _ in range(6):
        c = rng.uniform(-100, 100, 3)
        r = rng.uniform(6, 15)
        img[((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) < r * r] = 6.0
    return img.ravel(order="F").astype(np.float32)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock / throttle samples every 50 ms.  Started before the
    warm-up (nvidia-smi needs a few hundred ms to begin sampling), it keeps
    only the samples whose timestamps fall inside the timed region marked by
    mark_start() / mark_stop() (the nearest ones if none does)."""
    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_stop(self):
        self.t1 = time.time()

    @staticmethod
    def _epoch(ts):
        import datetime
        try:
            return datetime.datetime.strptime(ts.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 10:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        if self.t0 is not None and self.t1 is not None:
            stamped = [(self._epoch(r[0]), r) for r in rows]
            inside = [r for t, r in stamped if t is not None and self.t0 - 0.05 <= t <= self.t1 + 0.05]
            if not inside:
                near = sorted((abs(t - 0.5 * (self.t0 + self.t1)), i) for i, (t, r) in enumerate(stamped)
                              if t is not None)
                inside = [stamped[i][1] for _, i in near[:2]]
            rows = inside or rows
        rows = [r[1:] for r in rows]  # drop the timestamp
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# cone-beam CT workload
# ---------------------------------------------------------------------------

def cbct_options(small=False, views=None):
    from omega_b200.projector import proj
    o = proj.projectorClass()
    panel, nproj, n = (128, 90, 64) if small else (512, 360, 256)
    nproj = views or nproj
    o.CT = True
    o.nRowsD = o.nColsD = panel
    o.nProjections = nproj
    o.dPitchX = o.dPitchY = 0.4 * (512 // panel)
    o.sourceToCRot, o.sourceToDetector = 500., 1000.
    o.Nx = o.Ny = o.Nz = n
    o.FOVa_x = o.FOVa_y = o.axial_fov = 64.
    o.angles = np.linspace(0, 2 * np.pi, nproj, endpoint=False).astype(np.float32)
    o.projector_type = 5
    o.subsets, o.subsetType = 1, 8
    o.PDHG, o.TV = True, True
    o.beta, o.TVsmoothing = 0.05, 1e-4
    o.verbose = 0
    o.SinM = np.zeros((panel, panel, nproj), dtype=np.float32)  # marks projection data (not list-mode)
    o.addProjector()
    o.SinM = np.empty(0, dtype=np.float32)
    return o


def shepp_logan_3d(o, seed=7):
    """Seeded 3-D ellipsoid phantom, attenuation 0-0.02 /mm: the ten
    ellipsoids of the 3-D Shepp-Logan layout with randomly jittered centres."""
    rng = np.random.default_rng(seed)
    n = int(o.Nx[0])
    c = (np.arange(n, dtype=np.float32) + 0.5) / n * 2 - 1
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    # (mu, a, b, c, x0, y0, z0, phi) in units of the half FOV
    E = [(0.020, .69, .92, .81, 0, 0, 0, 0), (-0.016, .6624, .874, .78, 0, -.0184, 0, 0),
         (-0.004, .11, .31, .22, .22, 0, 0, -18), (-0.004, .16, .41, .28, -.22, 0, 0, 18),
         (0.002, .21, .25, .41, 0, .35, -.15, 0), (0.002, .046, .046, .05, 0, .1, .25, 0),
         (0.002, .046, .046, .05, 0, -.1, .25, 0), (0.002, .046, .023, .05, -.08, -.605, 0, 0),
         (0.002, .023, .023, .02, 0, -.606, 0, 0), (0.002, .023, .046, .02, .06, -.605, 0, 0)]
    img = np.zeros((n, n, n), dtype=np.float32)
    for mu, a, b, cc, x0, y0, z0, phi in E:
        x0, y0, z0 = np.array([x0, y0, z0]) + rng.uniform(-0.01, 0.01, 3)
        t = np.radians(phi)
        xr = (X - x0) * np.cos(t) + (Y - y0) * np.sin(t)
        yr = -(X - x0) * np.sin(t) + (Y - y0) * np.cos(t)
        img[(xr / a) ** 2 + (yr / b) ** 2 + ((Z - z0) / cc) ** 2 <= 1] += mu
    return np.clip(img, 0, 0.02).ravel(order="F")


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def choose_tuning(o, args, n_frames):
    """The autotuner's launch shapes, or the ones given with --tuning."""
    if args.tuning:
        o.tuning = {k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))}
        return o.tuning
    return o.autotune(n_frames=n_frames, repeats=2)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return ""


class Timed:
    """Per-step CUDA-event timing of named phases on one stream."""

    def __init__(self, stream):
        import torch
        self.torch = torch
        self.stream = stream
        self.events = []

    def mark(self):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        self.events.append(e)

    def phases(self):
        self.events[-1].synchronize()
        out = [a.elapsed_time(b) / 1e3 for a, b in zip(self.events[:-1], self.events[1:])]
        self.events = []
        return out


def max_over_ranks(values, device=None):
    """The slowest rank's times (omega_b200.distributed.max_over_ranks)."""
    from omega_b200.distributed import max_over_ranks as m
    return m(values, device=device)


def run_timed(args, world, dev, step, n_phases):
    """Warm-up, then exactly args.steps steps bracketed by barrier + sync,
    with an L2 flush between steps outside the events.  Returns per-phase
    totals (seconds), the clock record and the wall time."""
    import torch
    import torch.distributed as dist
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev)
    tm = Timed(stream)
    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    for _ in range(max(args.warmup, 0)):
        step(tm)
        tm.phases()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    tot = [0.0] * n_phases
    clocks.mark_start()
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        step(tm)
        for i, t in enumerate(tm.phases()):
            tot[i] += t
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clocks.mark_stop()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
        tot = max_over_ranks(tot, device=dev)
    return tot, clk, wall


def e2e_time(args, world, dev, step_host):
    import torch
    import torch.distributed as dist
    stream = torch.cuda.current_stream(dev)
    times = []
    for it in range(args.warmup + args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_host()
        e1.record(stream)
        e1.synchronize()
        if it >= args.warmup:
            times.append(e0.elapsed_time(e1) / 1e3)
    total = sum(times)
    if world > 1:
        total = max_over_ranks([total], device=dev)[0]
    return total


def roofline(name, model_bytes, duration, traffic_key, compulsory_bytes=None, launches=1):
    """HBM roofline of the dominant kernel.  ``achieved`` / ``frac`` count the
    DRAM bytes the kernel really moves per call: the ncu dram__bytes of one
    launch (profiles/, scaled to the full workload as the summary states)
    times the launches of the timed phase, over its event-timed duration.
    ``model_*`` keep the survey's cache-less byte model (every tap a DRAM
    access, above 1 when taps hit on chip) and ``compulsory_*`` the bytes any
    implementation must move (inputs and outputs once)."""
    peak, src = measured_peak()
    traffic = PROFILED_TRAFFIC.get(traffic_key)
    out = {"bound": "hbm", "kernel": name, "peak": peak, "unit": "GB/s", "peak_source": src,
           "model_bytes": model_bytes, "model_achieved": model_bytes / duration / 1e9,
           "model_frac": model_bytes / duration / 1e9 / peak, "limiter": PROFILED_LIMITER.get(traffic_key)}
    if traffic is not None:
        achieved = traffic * launches / duration / 1e9
        out.update({"achieved": achieved, "frac": achieved / peak, "traffic": traffic,
                    "basis": f"DRAM bytes ncu counted per launch x {launches} launch(es) / event-timed phase"})
    else:
        out.update({"achieved": out["model_achieved"], "frac": out["model_frac"], "traffic": None,
                    "basis": "no ncu capture of this workload: cache-less byte model"})
    if compulsory_bytes is not None:
        out["compulsory_bytes"] = compulsory_bytes
        out["compulsory_frac"] = compulsory_bytes / duration / 1e9 / peak
    return out


# ---------------------------------------------------------------------------
# our arm: cone-beam CT, one PDHG+TV iteration per step
# ---------------------------------------------------------------------------


I0 = 1e5


def cbct_sample_geometry(o, n_views):
    """Oracle geometry restricted to the first n_views projections."""
    from oracle import oracle as orc
    g = orc.Geometry(o)
    g.n_meas = np.array([0, n_views], dtype=np.int64)
    g.n_subsets = 1
    return g


def cbct_cpu_rate(o, image, seconds, views_per_call=4):
    """FP64 OpenMP restatement of the type-5 pair (there is no reference CPU
    code for projector type 5) on a bounded sample of projections, repeated
    for about `seconds`; returns rays/s of FP+BP pairs and the sample."""
    from oracle import oracle as orc
    g = cbct_sample_geometry(o, views_per_call)
    rays = g.rays(0)
    done, t0 = 0, time.perf_counter()
    while True:
        y = orc.bdd_forward(g, image, 0)
        orc.bdd_backward(g, y, 0)
        done += rays
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return done / el, f"{views_per_call} of {int(o.nProjections)} projections ({rays} rays) per FP+BP pair, " \
                      f"{done // rays} pairs in {el:.1f} s"


def learned_time_to_logl(studies=8, timing_studies=4):
    """Time to the plain 20-iteration OSEM log-likelihood, learned warm start
    vs plain OSEM, on held-out seeded studies of the dynamic-PET geometry
    (16 subsets), with the committed network weights."""
    import torch
    from omega_b200 import warmstart as ws
    path = os.path.join(ROOT, "omega_b200", "weights", "warmstart_pet128.npz")
    state = dict(np.load(path))
    o = ws.pet_geometry()
    o.initProj()
    o.autotune(n_frames=studies, repeats=1)
    summary, _ = ws.evaluate(o, state, 3_000_000, studies, (1e7, 1e8), converged=20, batch=studies,
                             timing_studies=timing_studies)
    torch.cuda.synchronize()
    return {"studies": summary["studies"], "reached_plain_L20": summary["reached_L20"],
            "continuation_iterations_median": summary["k_median"], "continuation_iterations_max": summary["k_max"],
            "plain_20_iterations_ms": summary["plain_ms_median"], "warm_start_ms": summary["warm_ms_median"],
            "time_ratio": summary["time_ratio_median"],
            "timed_continuation_iterations": summary["timed_continuation"],
            "timed_studies": summary["timed_studies"], "timed_reached_plain_L20": summary["timed_reached_L20"],
            "rel_l2_warm_vs_plain20": summary["rel_l2_warm_vs_plain20_median"],
            "setup": "384 crystals x 32 rings, 128x128x63 image, 16 subsets, 1e7-1e8 counts; timed warm path = 2 "
                     "OSEM iterations + BF16 U-Net + a fixed 4 OSEM iterations + the log-likelihood check, the "
                     "same for every study (no per-study stop count); plain = 20 iterations; CUDA events per "
                     "study",
            "weights": "omega_b200/weights/warmstart_pet128.npz (5000 training studies)"}


def run_cbct(args, rank, world, dev):
    import torch
    from omega_b200 import _native
    from omega_b200 import reconstruction as rec
    small = args.workload == "cbct_small"
    o = cbct_options(small, args.views)
    o.initProj()
    h = o._handle
    n = int(o.N[0])
    m = o.measurementCount(-1)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    # data: Poisson transmission counts at I0, zeros clamped to 1, log(I0/I)
    mu_host = shepp_logan_3d(o)
    mu = torch.from_numpy(mu_host).to(dev)
    yc = torch.empty(m, device=dev)
    _native.call("omb_forward", h, -1, P(mu), P(yc), sp)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    counts = torch.poisson(I0 * torch.exp(-yc), generator=gen).clamp_(min=1.0)
    y = torch.log(I0 / counts)
    del counts, yc
    tuning = choose_tuning(o, args, 1)
    tau = 1.0 / rec.power_method(o, 20, seed=0)
    sigma, theta = 1.0, 1.0
    beta, smooth = float(o.beta), float(o.TVsmoothing)

    x = torch.full((n,), 1e-4, device=dev)
    bufs = [x, torch.empty_like(x)]
    u = x.clone()
    p = torch.zeros(m, device=dev)
    wm = torch.empty(m, device=dev)
    wi = torch.empty(n, device=dev)

    def step(tm):
        a, b = bufs
        tm.mark()
        _native.call("omb_forward", h, -1, P(a), P(wm), sp)
        tm.mark()
        _native.call("omb_pdhg_dual", P(p), P(wm), P(y), m, sigma, sp)
        tm.mark()
        _native.call("omb_backward", h, -1, P(p), P(wi), None, 0, sp)
        tm.mark()
        _native.call("omb_pdhg_primal", h, P(a), P(wi), P(u), P(b), tau, theta, beta, smooth, 1, sp)
        tm.mark()
        bufs.reverse()

    tot, clk, wall = run_timed(args, world, dev, step, 4)
    t_fp, t_dual, t_bp, t_primal = tot
    total = sum(tot)

    # end to end: the iterate copied in from pinned host memory, one fused
    # omb_pdhg_iteration, the new iterate copied out
    h_in = torch.full((n,), 1e-4).pin_memory()
    h_out = torch.empty(n, dtype=torch.float32).pin_memory()

    def step_host():
        a, b = bufs
        a.copy_(h_in, non_blocking=True)
        _native.call("omb_pdhg_iteration", h, P(a), P(b), P(u), P(p), P(y), tau, sigma, theta, beta, smooth, 1,
                     P(wm), P(wi), sp)
        h_out.copy_(b, non_blocking=True)

    e2e_total = e2e_time(args, world, dev, step_host)

    # the ray-driven (scatter) backprojection of the same dual variable, the
    # exact adjoint of the forward projection, timed beside the gather
    ray_ms = []
    for it in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _native.call("omb_backward", h, -1, P(p), P(wi), None, _native.OMB_BP_RAY, sp)
        e1.record(stream)
        e1.synchronize()
        if it:
            ray_ms.append(e0.elapsed_time(e1))
    if rank != 0:
        return None
    K = args.steps
    value = m * K * world / total
    nproj = int(o.nProjections)
    slices = int(o.Nx[0])  # every ray crosses all slices of its main axis (Nx = Ny here)
    fp_bytes = m * (slices * 16 + 4)
    bp_bytes = n * nproj * 16 + n * 4
    mean_fp, mean_bp = t_fp / K, t_bp / K
    if mean_bp >= mean_fp:
        rl = roofline("bdd_bp", bp_bytes, mean_bp, (args.workload, "bdd_bp"), (n + m) * 4)
    else:
        rl = roofline("bdd_fp", fp_bytes, mean_fp, (args.workload, "bdd_fp"), (n + m) * 4)
    rl["model"] = ("cache-less tap bytes: FP = rays x (slices x 4 taps x 4 B + 4 B out); BP = voxels x views x "
                   "4 taps x 4 B + 4 B out. The 67 MB volume is L2-resident, so the taps are served on chip")
    panel = int(o.nRowsD)
    line = {
        "metric": "proj+backproj rays/s", "value": value, "unit": "rays/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * total / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 3-D ellipsoid phantom, Poisson transmission counts at I0=1e5)",
        "config": {"workload": (f"cone-beam CT, {panel}x{panel} panel 0.4 mm, {nproj} views over 360 deg, "
                                "SOD 500 / SDD 1000 mm, 256^3 volume 0.25 mm, branchless distance-driven (type 5), "
                                "one PDHG+TV iteration per step") if not small else
                   "cone-beam CT small (128^2 panel, 90 views, 64^3) for profiling",
                   "rays_per_step": m, "voxels": n, "views": nproj, "subsets": 1, "tuning": tuning,
                   "parallelism": f"replicas x{world}",
                   "l2": "256 MB L2 flush between steps; the measurement vectors (%.0f MB each) exceed L2"
                         % (m * 4 / 1e6)},
        "fp_ms": 1e3 * mean_fp, "bp_ms": 1e3 * mean_bp, "dual_ms": 1e3 * t_dual / K,
        "primal_tv_ms": 1e3 * t_primal / K, "tau": tau,
        "bp_ray": {"ms": statistics.median(ray_ms),
                   "what": "ray-driven scatter backprojection (float atomics), the exact adjoint of the forward "
                           "projection, of the same data; not part of the step"},
        "roofline": rl,
        "e2e": {"value": m * K * world / e2e_total, "unit": "rays/s", "h2d_bytes_per_step": n * 4,
                "d2h_bytes_per_step": n * 4,
                "what": "each step copies the iterate (%.0f MB) host->device and the new iterate back; the "
                        "measurement vector (%.0f MB) stays resident across iterations, as in an iterative "
                        "reconstruction" % (n * 4 / 1e6, m * 4 / 1e6)},
        "gpu_launches": 5 * K,
        "clocks": clk,
        "wall_s": wall,
    }
    if not args.no_learned and world == 1 and not small:
        try:
            line["time_to_logl"] = learned_time_to_logl()
        except Exception as e:  # must not hide the projector number
            line["time_to_logl"] = {"error": str(e)}
    if not args.no_baseline and world == 1:
        try:
            v, sample = cbct_cpu_rate(o, mu_host, 10.0)
            line["cpu_baseline"] = {"value": v, "unit": "rays/s", "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": sample + "; FP64 OpenMP restatement (the reference has no CPU "
                                              f"type-5 projector); host CPU {cpu_model()}"}
        except Exception as e:  # baseline failures must not hide the GPU number
            line["cpu_baseline"] = {"error": str(e)}
    return line


# ---------------------------------------------------------------------------
# our arm: dynamic PET, FP of all frames then BP of all frames per step
# ---------------------------------------------------------------------------

def dynpet_cpu_rate(o, image, seconds):
    from oracle import oracle as orc
    g = orc.Geometry(o)
    threads = os.cpu_count() or 1
    use_ref = orc.ref_lib() is not None
    rays = g.rays(0)
    done, t0 = 0, time.perf_counter()
    while True:
        if use_ref:
            yy = orc.ref_forward(g, image, 0, precision="float", threads=threads)
            orc.ref_backward(g, yy, 0, precision="float", threads=threads)
        else:
            yy = orc.forward(g, image, 0)
            orc.backward(g, yy, 0)
        done += rays
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    desc = "reference projectorType123Implementation4<float> (OpenMP)" if use_ref else "FP64 oracle restatement"
    return done / el, threads if use_ref else 1, "reference" if use_ref else "port", \
        f"frame 0, subset 0 ({g.n_meas[1] - g.n_meas[0]} sinograms, {rays} rays) per FP+BP pair, " \
        f"{done // rays} pairs in {el:.1f} s; {desc}"


def run_dynpet(args, rank, world, dev):
    import torch
    from omega_b200 import _native
    small = args.workload == "dynpet_small"
    frames = args.frames or (4 if small else 24)
    o = dynamic_pet_options(small)
    o.initProj()
    h = o._handle
    n = int(o.N[0])
    m = o.measurementCount(-1)
    imgs_host = dynamic_images(o, frames)
    imgs = torch.from_numpy(imgs_host).to(dev)
    ys = torch.empty((frames, m), device=dev)
    back = torch.empty((frames, n), device=dev)
    sp = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    def step(tm):
        tm.mark()
        _native.call("omb_forward_frames", h, -1, frames, P(imgs), n, P(ys), m, sp)
        tm.mark()
        _native.call("omb_backward_frames", h, -1, frames, P(ys), m, P(back), n, sp)
        tm.mark()

    tuning = choose_tuning(o, args, frames)
    npx = ctypes.c_int64()
    _native.call("omb_intersection_count", h, -1, ctypes.byref(npx), sp)
    sum_np = npx.value
    tot, clk, wall = run_timed(args, world, dev, step, 2)
    t_fp, t_bp = tot
    total = t_fp + t_bp

    h_in = torch.from_numpy(imgs_host).pin_memory()
    h_out = torch.empty((frames, n), dtype=torch.float32).pin_memory()

    class _NoMarks:
        def mark(self):
            pass

    def step_host():
        imgs.copy_(h_in, non_blocking=True)
        step(_NoMarks())
        h_out.copy_(back, non_blocking=True)

    e2e_total = e2e_time(args, world, dev, step_host)
    if rank != 0:
        return None
    K = args.steps
    ray_frames = m * frames
    fp_bytes = frames * (4 * sum_np + 32 * m)
    bp_bytes = frames * (8 * sum_np + 28 * m)
    mean_fp, mean_bp = t_fp / K, t_bp / K
    comp = frames * (n + m) * 4
    if mean_bp >= mean_fp:
        rl = roofline("siddon_bp", bp_bytes, mean_bp, (args.workload, "siddon_bp"), comp)
    else:
        rl = roofline("siddon_fp", fp_bytes, mean_fp, (args.workload, "siddon_fp"), comp)
    rl["model"] = "cache-less: FP = frames x sum_rays (4 Np + 32) B; BP = frames x sum_rays (8 Np + 28) B"
    line = {
        "metric": "proj+backproj rays/s", "value": ray_frames * K * world / total, "unit": "rays/s",
        "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * total / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded dynamic phantom, gamma-variate time-activity curves)",
        "config": {"workload": ("dynamic PET, 24 frames, 384 crystals x 32 rings, 256x192x63 sinograms, "
                                "128x128x63 image, improved Siddon FP+BP") if not small else
                   "dynamic PET small (8 rings) for profiling",
                   "frames": frames, "rays_per_frame": m, "intersections_per_frame": sum_np,
                   "subsets": int(o.subsets), "tuning": tuning, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (sinograms %.0f MB per step) plus a 256 MB L2 flush between steps"
                         % (frames * m * 4 / 1e6)},
        "fp_ms": 1e3 * mean_fp, "bp_ms": 1e3 * mean_bp,
        "roofline": rl,
        "e2e": {"value": ray_frames * K * world / e2e_total, "unit": "rays/s",
                "h2d_bytes_per_step": frames * n * 4, "d2h_bytes_per_step": frames * n * 4},
        "gpu_launches": 2 * K,
        "clocks": clk,
        "wall_s": wall,
    }
    if not args.no_baseline and world == 1:
        try:
            v, cores, kind, sample = dynpet_cpu_rate(o, imgs_host[0], 10.0)
            line["cpu_baseline"] = {"value": v, "unit": "rays/s", "cores": cores, "kind": kind,
                                    "sample": sample + f"; host CPU {cpu_model()}"}
        except Exception as e:
            line["cpu_baseline"] = {"error": str(e)}
    return line


def tube_cpu_rate(o, image, seconds):
    """The reference's own CPU projector with projector type 2 (FP64, OpenMP) on subset 0, else the FP64
    restatement."""
    from oracle import oracle as orc
    g = orc.Geometry(o)
    threads = os.cpu_count() or 1
    use_ref = orc.ref_lib() is not None
    rays = g.rays(0)
    done, t0 = 0, time.perf_counter()
    while True:
        if use_ref:
            yy = orc.ref_orth(g, image, 0, True, 2, threads=threads)
            orc.ref_orth(g, yy, 0, False, 2, threads=threads)
        else:
            yy = orc.orth_forward(g, image, 0)
            orc.orth_backward(g, yy, 0)
        done += rays
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    desc = "reference projectorType123Implementation4<double> with the orthogonal-distance tube (OpenMP)" \
        if use_ref else "FP64 oracle restatement"
    return done / el, threads if use_ref else 1, "reference" if use_ref else "port", \
        f"subset 0 ({rays} rays) per FP+BP pair, {done // rays} pairs in {el:.1f} s; {desc}"


def run_tube(args, rank, world, dev):
    """Projector type 2 (orthogonal-distance tube, 4 mm) on the dynamic-PET
    scanner, one frame: the 16 subsets projected forward, then back, each
    through the resident system matrix of its tube weights (built by the
    warm-up)."""
    import torch
    from omega_b200 import _native
    small = args.workload == "tube_small"
    o = dynamic_pet_options(small)
    o.projector_type = 2
    o.tube_width_z = o.tube_width_xy = 4.0
    o.addProjector()
    o.initProj()
    h = o._handle
    n = int(o.N[0])
    S = int(o.subsets)
    ms = [int(o.measurementCount(s)) for s in range(S)]
    m = sum(ms)
    img_host = dynamic_images(o, 1)[0]
    x = torch.from_numpy(np.ascontiguousarray(img_host)).to(dev)
    ys = [torch.empty(ms[s], device=dev) for s in range(S)]
    back = torch.empty(n, device=dev)
    sp = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    tuning = {"siddon_bp_matrix": 1}
    if args.tuning:
        tuning.update({k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))})
    o.tuning = tuning

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    live = [s for s in range(S) if ms[s] > 0]   # the small geometry leaves some subsets empty

    def step(tm):
        tm.mark()
        for s in live:
            _native.call("omb_forward_frames", h, s, 1, P(x), n, P(ys[s]), ms[s], sp)
        tm.mark()
        for s in live:
            _native.call("omb_backward_frames", h, s, 1, P(ys[s]), ms[s], P(back), n, sp)
        tm.mark()

    tot, clk, wall = run_timed(args, world, dev, step, 2)
    t_fp, t_bp = tot
    total = t_fp + t_bp
    h_in = torch.from_numpy(np.ascontiguousarray(img_host)).pin_memory()
    h_out = torch.empty(n, dtype=torch.float32).pin_memory()

    class _NoMarks:
        def mark(self):
            pass

    def step_host():
        x.copy_(h_in, non_blocking=True)
        step(_NoMarks())
        h_out.copy_(back, non_blocking=True)

    e2e_total = e2e_time(args, world, dev, step_host)
    if rank != 0:
        return None
    nnz = 0
    for s in live:
        v = ctypes.c_int64()
        _native.call("omb_system_matrix_nnz", h, s, ctypes.byref(v))
        nnz += v.value
    K = args.steps
    mean_fp, mean_bp = t_fp / K, t_bp / K
    # algorithmic bytes through the matrix: 8 bytes a weight plus the 4-byte gather it drives, and the
    # outputs once (FP: measurements; BP: one image a subset)
    fp_bytes = 12 * nnz + 4 * m
    bp_bytes = 12 * nnz + 4 * n * S
    comp = (n + m) * 4
    if mean_bp >= mean_fp:
        rl = roofline("tube_bp", bp_bytes, mean_bp, (args.workload, "tube_bp"), comp)
    else:
        rl = roofline("tube_fp", fp_bytes, mean_fp, (args.workload, "tube_fp"), comp)
    rl["model"] = "through the matrix: FP = 12 nnz + 4 m B; BP = 12 nnz + 4 N S B (nnz the tube weights)"
    line = {
        "metric": "proj+backproj rays/s", "value": m * K * world / total, "unit": "rays/s",
        "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * total / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantom)",
        "config": {"workload": ("PET, 384 crystals x 32 rings, 256x192x63 sinograms, 128x128x63 image, projector "
                                "type 2 (orthogonal-distance tube, 4 mm), 16 subsets, through the resident system "
                                "matrix") if not small else "tube small (8 rings) for profiling",
                   "rays_per_step": m, "tube_weights": nnz, "subsets": S, "tuning": tuning,
                   "parallelism": f"replicas x{world}", "l2": "256 MB L2 flush between steps"},
        "fp_ms": 1e3 * mean_fp, "bp_ms": 1e3 * mean_bp,
        "roofline": rl,
        "e2e": {"value": m * K * world / e2e_total, "unit": "rays/s", "h2d_bytes_per_step": n * 4,
                "d2h_bytes_per_step": n * 4},
        "gpu_launches": 2 * S * K,
        "clocks": clk,
        "wall_s": wall,
    }
    if not args.no_baseline and world == 1:
        try:
            v, cores, kind, sample = tube_cpu_rate(o, img_host, 10.0)
            line["cpu_baseline"] = {"value": v, "unit": "rays/s", "cores": cores, "kind": kind,
                                    "sample": sample + f"; host CPU {cpu_model()}"}
        except Exception as e:
            line["cpu_baseline"] = {"error": str(e)}
    return line


# ---------------------------------------------------------------------------
# our arm: 64 fan-beam CT slices of uneven sizes, one persistent launch per
# direction (omb_batch_forward / omb_batch_backward)
# ---------------------------------------------------------------------------

def fanbeam_items(small=False, seed=64):
    """Seeded slice sizes: n x n images, n in 128..512 (multiples of 16),
    180-720 views, ceil(1.5 n) detectors per view."""
    from omega_b200.projector.batch import fanbeam_slice
    rng = np.random.default_rng(seed)
    count = 8 if small else 64
    sizes = [(16 * int(rng.integers(8, 33)), int(rng.integers(180, 721))) for _ in range(count)]
    return [fanbeam_slice(n, v) for n, v in sizes], sizes


def run_fanbeam(args, rank, world, dev):
    import torch
    from omega_b200 import _native
    from omega_b200.projector.batch import ProjectorBatch
    small = args.workload == "fanbeam64_small"
    items, sizes = fanbeam_items(small)
    batch = ProjectorBatch(items)
    nimg, nmeas = int(batch.image_offsets[-1]), int(batch.measurement_offsets[-1])
    rng = np.random.default_rng(5)
    x_host = rng.uniform(0.0, 1.0, nimg).astype(np.float32)
    x = torch.from_numpy(x_host).to(dev)
    y = torch.empty(nmeas, device=dev)
    back = torch.empty(nimg, device=dev)
    sp = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    def step(tm):
        tm.mark()
        _native.call("omb_batch_forward", batch._handle, P(x), P(y), sp)
        tm.mark()
        _native.call("omb_batch_backward", batch._handle, P(y), P(back), sp)
        tm.mark()

    tot, clk, wall = run_timed(args, world, dev, step, 2)
    t_fp, t_bp = tot
    total = t_fp + t_bp
    K = args.steps
    # the same work with one launch pair per slice (separate handles)
    for o in items:
        o.initProj()
    npx = 0
    for o in items:
        c = ctypes.c_int64()
        _native.call("omb_intersection_count", o._handle, -1, ctypes.byref(c), sp)
        npx += c.value
    xs = [x[int(batch.image_offsets[i]):int(batch.image_offsets[i + 1])] for i in range(len(items))]
    ys = [y[int(batch.measurement_offsets[i]):int(batch.measurement_offsets[i + 1])] for i in range(len(items))]
    bs = [back[int(batch.image_offsets[i]):int(batch.image_offsets[i + 1])] for i in range(len(items))]

    def step_single(tm):
        tm.mark()
        for o, xi, yi in zip(items, xs, ys):
            _native.call("omb_forward", o._handle, -1, P(xi), P(yi), sp)
        tm.mark()
        for o, yi, bi in zip(items, ys, bs):
            _native.call("omb_backward", o._handle, -1, P(yi), P(bi), None, 0, sp)
        tm.mark()

    single, _, _ = run_timed(args, world, dev, step_single, 2)
    h_in = torch.from_numpy(x_host).pin_memory()
    h_out = torch.empty(nimg, dtype=torch.float32).pin_memory()

    def step_host():
        x.copy_(h_in, non_blocking=True)
        _native.call("omb_batch_forward", batch._handle, P(x), P(y), sp)
        _native.call("omb_batch_backward", batch._handle, P(y), P(back), sp)
        h_out.copy_(back, non_blocking=True)

    e2e_total = e2e_time(args, world, dev, step_host)
    if rank != 0:
        return None
    mean_fp, mean_bp = t_fp / K, t_bp / K
    fp_bytes = 4 * npx + 32 * nmeas
    bp_bytes = 8 * npx + 28 * nmeas
    if mean_bp >= mean_fp:
        rl = roofline("batch_siddon_bp", bp_bytes, mean_bp, (args.workload, "bp"), (nimg + nmeas) * 4)
    else:
        rl = roofline("batch_siddon_fp", fp_bytes, mean_fp, (args.workload, "fp"), (nimg + nmeas) * 4)
    line = {
        "metric": "proj+backproj rays/s", "value": nmeas * K * world / total, "unit": "rays/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * total / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform random images)",
        "config": {"workload": f"{len(items)} 2-D fan-beam CT slices of uneven sizes (n x n images, n 128-512; "
                               "180-720 views; ceil(1.5 n) detectors), improved Siddon, one persistent launch per "
                               "direction", "slices": len(items), "rays_per_step": nmeas, "voxels": nimg,
                   "intersections": npx, "sizes": sizes, "parallelism": f"replicas x{world}",
                   "l2": "256 MB L2 flush between steps"},
        "fp_ms": 1e3 * mean_fp, "bp_ms": 1e3 * mean_bp,
        "per_slice_launches_ms": 1e3 * sum(single) / K,
        "roofline": rl,
        "e2e": {"value": nmeas * K * world / e2e_total, "unit": "rays/s", "h2d_bytes_per_step": nimg * 4,
                "d2h_bytes_per_step": nimg * 4},
        "gpu_launches": 2 * K, "clocks": clk, "wall_s": wall,
    }
    if not args.no_baseline and world == 1:
        try:
            from oracle import oracle as orc
            g = orc.Geometry(items[0])
            xi = x_host[:int(batch.image_offsets[1])]
            done, t0 = 0, time.perf_counter()
            while time.perf_counter() - t0 < 10.0:
                orc.backward(g, orc.forward(g, xi, -1), -1)
                done += g.rays(-1)
            el = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": done / el, "unit": "rays/s", "cores": 1, "kind": "port",
                                    "sample": f"slice 0 ({sizes[0][0]}^2 image, {sizes[0][1]} views) FP+BP pairs for "
                                              f"{el:.1f} s; FP64 restatement of the type-1 projector (the reference's "
                                              f"CPU projector build here is PET-only); host CPU {cpu_model()}"}
        except Exception as e:
            line["cpu_baseline"] = {"error": str(e)}
    return line


# ---------------------------------------------------------------------------
# our arm: the precision workload, projector type 4 with 15 TOF bins
# ---------------------------------------------------------------------------

def interp_model_bytes(o, nbins):
    """Cache-less bytes of the type-4 forward projection, sum over rays of
    32 nSteps + 8 NB + 24 (8 texels per trilinear sample), with nSteps per
    ray as projectorType4.cl:467-482 counts them (FP64 here), and its
    backprojection, sum of 8 nSteps + 28 (nearest-voxel atomics)."""
    xy = np.asarray(o.x, dtype=np.float64).reshape(-1, 4)
    z = np.asarray(o.z, dtype=np.float64).reshape(-1, 2)
    b = np.array([float(o.bx[0]), float(o.by[0]), float(o.bz[0])])
    bmax = b + np.array([int(o.Nx[0]) * float(o.dx[0]), int(o.Ny[0]) * float(o.dy[0]), int(o.Nz[0]) * float(o.dz[0])])
    dL = float(np.float32(o.dL))
    steps = 0
    for k in range(z.shape[0]):
        s = np.stack([xy[:, 0], xy[:, 1], np.full(len(xy), z[k, 0])], 1)
        d = np.stack([xy[:, 2], xy[:, 3], np.full(len(xy), z[k, 1])], 1)
        v = d - s
        with np.errstate(divide="ignore", invalid="ignore"):
            t1, t2 = (b - s) / v, (bmax - s) / v
        t0 = np.nanmax(np.minimum(t1, t2), 1)
        te = np.nanmin(np.maximum(t1, t2), 1)
        L = np.linalg.norm(v, axis=1)
        ok = te > t0
        steps += int(np.sum(np.floor((te[ok] - t0[ok]) / (dL / L[ok])) + 1))
    rays = xy.shape[0] * z.shape[0]
    return steps, 32 * steps + (8 * nbins + 24) * rays, 8 * steps + 28 * rays


def run_interp_tof(args, rank, world, dev):
    import torch
    from omega_b200 import _native
    small = args.workload == "interp_tof_small"
    o = tof_pet_options(small, imageReadPrecision="bf16", use_64bit_atomics=True)
    o.initProj()
    h = o._handle
    n = int(o.N[0])
    S = int(o.subsets)
    nb = int(o.TOF_bins_used)
    ms = [o.measurementCount(s) for s in range(S)]      # all TOF bins
    offs = np.concatenate([[0], np.cumsum(ms)]).astype(np.int64)
    x_host = tof_phantom(o)
    x = torch.from_numpy(x_host).to(dev)
    y = torch.empty(int(offs[-1]), device=dev)
    back = torch.empty(n, device=dev)
    sp = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def P(t, off=0):
        return ctypes.c_void_p(t.data_ptr() + 4 * int(off))

    def step(tm):
        tm.mark()
        for s in range(S):
            _native.call("omb_forward", h, s, P(x), P(y, offs[s]), sp)
        tm.mark()
        for s in range(S):
            _native.call("omb_backward", h, s, P(y, offs[s]), P(back), None, 0, sp)
        tm.mark()

    tuning = choose_tuning(o, args, 1)
    tot, clk, wall = run_timed(args, world, dev, step, 2)
    t_fp, t_bp = tot

    # the int64 fixed-point backprojection of the same step, timed apart,
    # and checked bit-identical run to run
    def step64(tm):
        tm.mark()
        for s in range(S):
            _native.call("omb_backward", h, s, P(y, offs[s]), P(back), None, 1, sp)
        tm.mark()

    t64, _, _ = run_timed(args, world, dev, step64, 1)
    first = back.clone()
    step64(Timed(torch.cuda.current_stream(dev)))
    torch.cuda.synchronize()
    int64_identical = bool(torch.equal(first.view(torch.int32), back.view(torch.int32)))

    h_in = torch.from_numpy(x_host).pin_memory()
    h_out = torch.empty(n, dtype=torch.float32).pin_memory()

    class _NoMarks:
        def mark(self):
            pass

    def step_host():
        x.copy_(h_in, non_blocking=True)
        step(_NoMarks())
        h_out.copy_(back, non_blocking=True)

    e2e_total = e2e_time(args, world, dev, step_host)
    if rank != 0:
        return None
    K = args.steps
    lors = int(offs[-1]) // nb
    total = t_fp + t_bp
    mean_fp, mean_bp = t_fp / K, t_bp / K
    steps_total, fp_bytes, bp_bytes = interp_model_bytes(o, nb)
    comp = (n + int(offs[-1])) * 4
    if mean_bp >= mean_fp:
        rl = roofline("interp_bp", bp_bytes, mean_bp, (args.workload, "interp_bp"), comp, launches=S)
    else:
        rl = roofline("interp_fp", fp_bytes, mean_fp, (args.workload, "interp_fp"), comp, launches=S)
    rl["model"] = ("cache-less: FP = sum_rays (32 nSteps + 8 NB + 24) B (8 texels per trilinear sample); "
                   "BP = sum_rays (8 nSteps + 28) B (nearest-voxel atomics)")
    line = {
        "metric": "proj+backproj rays/s", "value": lors * K * world / total, "unit": "rays/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * total / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (bf16 image reads in the forward projection)",
        "data": "synthetic (seeded anthropomorphic-style ellipsoid phantom)",
        "config": {"workload": ("3-D TOF PET, 672 crystals x 55 rings, 400x336x109 sinograms x 15 TOF bins "
                                "(200 ps FWHM), 200x200x109 image, interpolation projector (type 4), BF16 image "
                                "reads, FP32 accumulation, all 16 subsets forward then back per step")
                   if not small else "3-D TOF PET small (11 rings) for profiling",
                   "lors_per_step": lors, "bins_per_step": int(offs[-1]), "tof_bins": nb, "samples_per_step": steps_total,
                   "subsets": S, "tuning": tuning, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (%.0f MB of TOF sinograms) plus a 256 MB L2 flush between steps"
                         % (int(offs[-1]) * 4 / 1e6)},
        "fp_ms": 1e3 * mean_fp, "bp_ms": 1e3 * mean_bp, "bp_int64_ms": 1e3 * t64[0] / K,
        "int64_bit_identical": int64_identical, "bins_per_s": int(offs[-1]) * K * world / total,
        "roofline": rl,
        "e2e": {"value": lors * K * world / e2e_total, "unit": "rays/s", "h2d_bytes_per_step": n * 4,
                "d2h_bytes_per_step": n * 4},
        "gpu_launches": 2 * S * K, "clocks": clk, "wall_s": wall,
    }
    if not args.no_baseline and world == 1:
        try:
            v, sample = interp_cpu_rate(small, x_host, 10.0)
            line["cpu_baseline"] = {"value": v, "unit": "rays/s", "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": sample + "; FP64 restatement (OpenMP forward, one-thread atomic "
                                              "backprojection) pinned to the reference's projectorType4.cl; the "
                                              f"reference has no CPU type-4 projector; host CPU {cpu_model()}"}
        except Exception as e:
            line["cpu_baseline"] = {"error": str(e)}
    return line


def interp_cpu_rate(small, image, seconds):
    """FP64 restatement of the type-4 TOF pair on one sinogram of the same
    scanner, repeated for at least `seconds`."""
    from oracle import oracle as orc
    o = tof_pet_options(small, subsets=int(22 if small else 109))
    g = orc.Geometry(o)
    rays = g.rays(0)
    done, t0 = 0, time.perf_counter()
    while True:
        yy = orc.interp_forward(g, image, 0)
        orc.interp_backward(g, yy, 0)
        done += rays
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return done / el, f"one sinogram ({rays} LORs x {g.nbins} TOF bins) per FP+BP pair, {done // rays} pairs in {el:.1f} s"


# ---------------------------------------------------------------------------
# reference arm: the CPU implementation of the same step on a bounded sample
# ---------------------------------------------------------------------------

def run_reference(args):
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    times = []
    if args.workload.startswith("cbct"):
        o = cbct_options(args.workload == "cbct_small", args.views)
        img = shepp_logan_3d(o)
        g = cbct_sample_geometry(o, 4)
        rays = g.rays(0)
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            y = orc.bdd_forward(g, img, 0)
            orc.bdd_backward(g, y, 0)
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
        kind, cores = "port", threads
        sample = (f"4 of {int(o.nProjections)} projections ({rays} rays) per step; FP64 OpenMP restatement of the "
                  "type-5 pair (the reference has no CPU type-5 projector)")
        workload = "cone-beam CT (same geometry as ours), FP+BP pair over a bounded sample of projections"
    elif args.workload.startswith("fanbeam"):
        items, sizes = fanbeam_items(args.workload == "fanbeam64_small")
        g = orc.Geometry(items[0])
        img = np.random.default_rng(5).uniform(0.0, 1.0, g.n_img)
        rays = g.rays(-1)
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            orc.backward(g, orc.forward(g, img, -1), -1)
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
        kind, cores = "port", 1
        sample = (f"slice 0 ({sizes[0][0]}^2 image, {sizes[0][1]} views, {rays} rays) per step; FP64 restatement of "
                  "the type-1 projector (the reference's CPU projector build here is PET-only)")
        workload = "64 fan-beam CT slices (same sizes as ours), FP+BP pair over slice 0"
    elif args.workload.startswith("tube"):
        o = dynamic_pet_options(args.workload == "tube_small")
        o.projector_type = 2
        o.tube_width_z = o.tube_width_xy = 4.0
        o.addProjector()
        img = dynamic_images(o, 1)[0]
        g = orc.Geometry(o)
        use_ref = orc.ref_lib() is not None
        rays = g.rays(0)
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            if use_ref:
                y = orc.ref_orth(g, img, 0, True, 2, threads=threads)
                orc.ref_orth(g, y, 0, False, 2, threads=threads)
            else:
                y = orc.orth_forward(g, img, 0)
                orc.orth_backward(g, y, 0)
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
        kind, cores = ("reference", threads) if use_ref else ("port", 1)
        sample = f"subset 0 ({rays} rays) per step, projector type 2 (4 mm tube)"
        workload = "PET tube projector type 2 (same geometry as ours), FP+BP pair over subset 0"
    else:
        o = dynamic_pet_options(args.workload == "dynpet_small")
        img = dynamic_images(o, 1)[0]
        g = orc.Geometry(o)
        use_ref = orc.ref_lib() is not None
        rays = g.rays(0)
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            if use_ref:
                y = orc.ref_forward(g, img, 0, precision="float", threads=threads)
                orc.ref_backward(g, y, 0, precision="float", threads=threads)
            else:
                y = orc.forward(g, img, 0)
                orc.backward(g, y, 0)
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
        kind, cores = ("reference", threads) if use_ref else ("port", 1)
        sample = f"frame 0, subset 0 ({rays} rays) per step"
        workload = "dynamic PET (same geometry as ours), FP+BP pair over frame 0, subset 0"
    value = rays * args.steps / sum(times)
    return {
        "impl": "reference", "metric": "proj+backproj rays/s", "value": value, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if kind == "reference"
        else "f64", "data": "synthetic",
        "config": {"workload": workload, "sample_rays_per_step": rays, "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": cores, "kind": kind,
                         "sample": sample + f"; host CPU {cpu_model()}"},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    runs = {"cbct": run_cbct, "fanbeam": run_fanbeam, "dynpet": run_dynpet, "interp_tof": run_interp_tof,
            "tube": run_tube}
    run = next(f for k, f in runs.items() if args.workload.startswith(k))
    line = run(args, rank, world, dev)
    if args.workload == "cbct" and world == 1 and not args.no_legs:
        # the other projectors of the path, each timed the same way: improved
        # Siddon (dynamic PET), interpolation with TOF (precision workload) and
        # the orthogonal-distance tube (type 2)
        import copy

        import torch
        legs = {}
        for name, wl, fn in (("siddon_dynpet", "dynpet", run_dynpet), ("interp_tof", "interp_tof", run_interp_tof),
                             ("tube", "tube", run_tube)):
            torch.cuda.empty_cache()
            a = copy.copy(args)
            a.workload = wl
            a.tuning = None
            try:
                legs[name] = fn(a, rank, world, dev)
            except Exception as e:  # a leg must not hide the headline number
                legs[name] = {"error": f"{type(e).__name__}: {e}"}
        line["legs"] = legs
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
