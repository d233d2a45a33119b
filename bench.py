#!/usr/bin/env python
"""Projector throughput benchmark (one JSON line on rank 0).

Workload (default ``dynpet``): the batching PET study -- a 384-crystal x 32-ring
scanner (600 mm ring), 256 radial x 192 angle x 63 plane sinograms
(3,096,576 rays per frame), a 128 x 128 x 63 image over 300 x 300 x 126 mm,
24 frames of a dynamic study, improved Siddon (projector type 1), 16 subsets
of whole sinograms.  One step = forward projection of all 24 frames followed
by backprojection of the 24 resulting sinograms (every ray of every frame
once forward and once back), as one launch each.

metric: rays/s of FP+BP pairs (ray-frames forward- and back-projected per
second).  ``value`` times device-resident inputs with CUDA events; ``e2e``
times the same step through the C-ABI with pinned host images copied in and
the backprojected images copied out.  ``cpu_baseline`` is the reference's own
OpenMP CPU projector (projector_functions.h:1312, built into oracle/_ref) on
a bounded sample of the same workload.

--impl reference times that reference CPU projector alone (all host threads)
on the same metric; under torchrun only rank 0 runs it.
Multi-GPU: replicas (each rank projects its own 24-frame batch; no
collective on the data path); value = all ranks' ray-frames / max rank time.
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
# workload by rays; see profiles/ for the captures they come from.
PROFILED_TRAFFIC = {}
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="dynpet", choices=["dynpet", "dynpet_small"])
    p.add_argument("--frames", type=int, default=None)
    p.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline leg")
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


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

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
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own OpenMP projector on a bounded sample
# ---------------------------------------------------------------------------

def cpu_baseline(o, image, seconds=10.0):
    from oracle import oracle as orc
    g = orc.Geometry(o)
    threads = os.cpu_count() or 1
    use_ref = orc.ref_lib() is not None
    subset = 0
    rays = g.rays(subset)
    done = 0
    t0 = time.perf_counter()
    while True:
        if use_ref:
            y = orc.ref_forward(g, image, subset, precision="float", threads=threads)
            orc.ref_backward(g, y, subset, precision="float", threads=threads)
        else:
            y = orc.forward(g, image, subset)
            orc.backward(g, y, subset)
        done += rays
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    cpu_model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    cpu_model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"value": done / el, "unit": "rays/s", "cores": threads if use_ref else 1,
            "kind": "reference" if use_ref else "port",
            "sample": f"frame 0, subset 0 ({g.n_meas[1] - g.n_meas[0]} sinograms, {rays} rays), FP+BP pairs "
                      f"repeated for {el:.1f} s; {'reference projectorType123Implementation4<float> (OpenMP)' if use_ref else 'FP64 oracle restatement'}"
                      f"; host CPU {cpu_model}"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from omega_b200 import _native
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    small = args.workload == "dynpet_small"
    frames = args.frames or (4 if small else 24)
    o = dynamic_pet_options(small)
    o.initProj()
    L = _native.lib()
    h = o._handle
    n = int(o.N[0])
    m = o.measurementCount(-1)
    rays_per_frame = m
    imgs_host = dynamic_images(o, frames)
    imgs = torch.from_numpy(imgs_host).to(dev)
    ys = torch.empty((frames, m), device=dev)
    back = torch.empty((frames, n), device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev)

    def step():
        _native.call("omb_forward_frames", h, -1, frames, ctypes.c_void_p(imgs.data_ptr()), n,
                     ctypes.c_void_p(ys.data_ptr()), m, sp)
        ev_mid.record(stream)
        _native.call("omb_backward_frames", h, -1, frames, ctypes.c_void_p(ys.data_ptr()), m,
                     ctypes.c_void_p(back.data_ptr()), n, sp)

    ev_mid = torch.cuda.Event(enable_timing=True)
    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    # total voxel intersections of one frame (for the algorithmic-byte model)
    npx = ctypes.c_int64()
    _native.call("omb_intersection_count", h, -1, ctypes.byref(npx), sp)
    sum_np = npx.value

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    t_fp, t_bp = [], []
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        ev_mid = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e2.record(stream)
        e2.synchronize()
        t_fp.append(e0.elapsed_time(ev_mid) / 1e3)
        t_bp.append(ev_mid.elapsed_time(e2) / 1e3)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    t_step = [a + b for a, b in zip(t_fp, t_bp)]
    total = sum(t_step)
    if world > 1:
        tt = torch.tensor([total], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total = float(tt.item())

    # end to end through the C-ABI: pinned host images in, backprojections out
    h_in = torch.from_numpy(imgs_host).pin_memory()
    h_out = torch.empty((frames, n), dtype=torch.float32).pin_memory()
    e2e_times = []
    for it in range(args.warmup + args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        imgs.copy_(h_in, non_blocking=True)
        step()
        h_out.copy_(back, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if it >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1) / 1e3)
    e2e_total = sum(e2e_times)
    if world > 1:
        tt = torch.tensor([e2e_total], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_total = float(tt.item())

    if rank != 0:
        return None
    ray_frames = rays_per_frame * frames
    value = ray_frames * args.steps * world / total
    # roofline of the dominant kernel (algorithmic bytes per launch / its mean duration)
    fp_bytes = frames * (4 * sum_np + 32 * rays_per_frame)
    bp_bytes = frames * (8 * sum_np + 28 * rays_per_frame)
    mean_fp, mean_bp = sum(t_fp) / len(t_fp), sum(t_bp) / len(t_bp)
    name, nbytes, dur = ("siddon_bp", bp_bytes, mean_bp) if mean_bp >= mean_fp else ("siddon_fp", fp_bytes, mean_fp)
    peak, peak_src = FALLBACK_HBM_GBS, "fallback"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        pass
    achieved = nbytes / dur / 1e9
    traffic = PROFILED_TRAFFIC.get((args.workload, name))
    line = {
        "metric": "proj+backproj rays/s", "value": value, "unit": "rays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded dynamic phantom, gamma-variate time-activity curves)",
        "config": {"workload": ("dynamic PET, 24 frames, 384 crystals x 32 rings, 256x192x63 sinograms, "
                                "128x128x63 image, improved Siddon FP+BP") if not small else
                   "dynamic PET small (8 rings) for profiling",
                   "frames": frames, "rays_per_frame": rays_per_frame, "intersections_per_frame": sum_np,
                   "subsets": int(o.subsets), "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (sinograms %.0f MB per step) plus a 256 MB L2 flush between steps"
                         % (frames * m * 4 / 1e6)},
        "fp_ms": 1e3 * mean_fp, "bp_ms": 1e3 * mean_bp,
        "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src,
                     "algorithmic_bytes": nbytes, "traffic": traffic},
        "e2e": {"value": ray_frames * args.steps * world / e2e_total, "unit": "rays/s",
                "h2d_bytes_per_step": frames * n * 4, "d2h_bytes_per_step": frames * n * 4},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
        "wall_s": wall,
    }
    if not args.no_baseline and world == 1:
        try:
            line["cpu_baseline"] = cpu_baseline(o, imgs_host[0])
        except Exception as e:  # baseline failures must not hide the GPU number
            line["cpu_baseline"] = {"error": str(e)}
    return line


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference(args):
    from oracle import oracle as orc
    small = args.workload == "dynpet_small"
    o = dynamic_pet_options(small)
    frames = args.frames or (4 if small else 24)
    img = dynamic_images(o, 1)[0]
    g = orc.Geometry(o)
    use_ref = orc.ref_lib() is not None
    threads = os.cpu_count() or 1
    subset = 0
    rays = g.rays(subset)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        if use_ref:
            y = orc.ref_forward(g, img, subset, precision="float", threads=threads)
            orc.ref_backward(g, y, subset, precision="float", threads=threads)
        else:
            y = orc.forward(g, img, subset)
            orc.backward(g, y, subset)
        if it >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = rays * args.steps / sum(times)
    kind = "reference" if use_ref else "port"
    return {
        "impl": "reference", "metric": "proj+backproj rays/s", "value": value, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "dynamic PET (same geometry as ours); each step one FP+BP pair over frame 0, "
                               "subset 0 (bounded sample)", "frames_full_workload": frames,
                   "sample_rays_per_step": rays, "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": threads if use_ref else 1, "kind": kind,
                         "sample": f"frame 0, subset 0 ({rays} rays) per step"},
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
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
