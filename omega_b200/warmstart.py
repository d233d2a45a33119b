"""Learned OSEM warm start: training data, training and the time-to-logL
comparison against plain OSEM.

Geometry: the dynamic-PET scanner (384 crystals x 32 rings, 600 mm ring,
256 x 192 x 63 span-3 sinograms, 128 x 128 x 63 image over a 300 mm FOV,
improved Siddon, 16 subsets).  Each study is a seeded phantom -- an
elliptic-cylinder body with 3-8 hot or cold ellipsoids and spheres -- whose
Siddon forward projection is scaled to a total count drawn log-uniformly
from `counts` and Poisson-sampled.  OSEM runs batched (all studies of a
batch share each ray walk, omb_osem_subset_frames) from a uniform image; the
network input is the 2-iteration image plus the sensitivity image, its
target the 20-iteration image.

Evaluation per held-out study: plain OSEM for 20 iterations gives the
target log-likelihood L20; the warm start runs 2 iterations, the network,
then plain OSEM iterations until its log-likelihood reaches L20 (at most
20).  Both paths are timed with CUDA events, and both images are compared
with a converged plain solution (`converged` iterations).

    python -m omega_b200.warmstart --train 5000 --eval 200 --minutes 5 --out weights.npz --report report.json
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time

import numpy as np

from . import _native
from . import reconstruction as rec
from .learned import UNet3D


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def pet_geometry(rings=32, subsets=16):
    """The dynamic-PET scanner with `subsets` whole-sinogram subsets."""
    from .projector import geometry as geo
    from .projector import proj
    o = proj.projectorClass()
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
    o.subsets, o.subsetType = subsets, 8
    o.verbose = 0
    o.addProjector()
    return o


def phantoms(o, first_seed, n, device):
    """n seeded phantoms (n, Nx*Ny*Nz) FP32 on `device`, Fortran order."""
    import torch
    nx, ny, nz = int(o.Nx[0]), int(o.Ny[0]), int(o.Nz[0])
    dx, dz = float(o.dx[0]), float(o.dz[0])
    xs = torch.arange(nx, device=device, dtype=torch.float32) * dx + (float(o.bx[0]) + 0.5 * dx)
    zs = torch.arange(nz, device=device, dtype=torch.float32) * dz + (float(o.bz[0]) + 0.5 * dz)
    Z, Y, X = torch.meshgrid(zs, xs, xs, indexing="ij")  # [z][y][x]: Fortran order when flattened
    out = torch.empty((n, nx * ny * nz), device=device)
    zc = 0.5 * (float(zs[0]) + float(zs[-1]))
    for k in range(n):
        rng = np.random.default_rng(first_seed + k)
        a, b = rng.uniform(70, 120), rng.uniform(55, 105)
        th = rng.uniform(0, np.pi)
        half_z = rng.uniform(0.35, 0.5) * nz * dz
        c, s = math.cos(th), math.sin(th)
        u = (X * c + Y * s) / a
        v = (-X * s + Y * c) / b
        body = ((u * u + v * v) <= 1.0) & ((Z - zc).abs() <= half_z)
        base = rng.uniform(0.5, 1.5)
        img = body.float() * base
        for _ in range(rng.integers(3, 9)):
            r = rng.uniform(6, 28, 3) if rng.random() < 0.6 else np.full(3, rng.uniform(6, 22))
            rho, phi = rng.uniform(0, 0.65), rng.uniform(0, 2 * np.pi)
            cx = rho * a * math.cos(phi) * c - rho * b * math.sin(phi) * s
            cy = rho * a * math.cos(phi) * s + rho * b * math.sin(phi) * c
            cz = zc + rng.uniform(-0.7, 0.7) * half_z
            e = ((X - cx) / r[0]) ** 2 + ((Y - cy) / r[1]) ** 2 + ((Z - cz) / r[2]) ** 2 <= 1.0
            level = rng.uniform(1.5, 5.0) if rng.random() < 0.7 else rng.uniform(0.0, 0.4)
            img = torch.where(e & body, img.new_full((), base * level), img)
        out[k] = img.reshape(-1)
    return out


def simulate(o, truth, counts, first_seed):
    """Poisson measurements (F, nTotMeas) of the phantoms, each scaled to its count."""
    import torch
    F, n = truth.shape
    M = o.measurementCount(-1)
    y = torch.empty((F, M), device=truth.device)
    st = ctypes.c_void_p(torch.cuda.current_stream(truth.device).cuda_stream)
    _native.call("omb_forward_frames", o._handle, -1, F, _ptr(truth), n, _ptr(y), M, st)
    scale = torch.as_tensor(counts, dtype=torch.float32, device=truth.device) / y.sum(dim=1).clamp_min(1e-12)
    g = torch.Generator(device=truth.device)
    g.manual_seed(int(first_seed))
    return torch.poisson(y * scale[:, None], generator=g)


def loglik_frames(o, x, m, work):
    """Poisson log-likelihood (FP64, device) of each study's image x[f]."""
    import torch
    F, n = x.shape
    M = m.shape[1]
    st = ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
    fp = work[: F * M]
    _native.call("omb_forward_frames", o._handle, -1, F, _ptr(x), n, _ptr(fp), M, st)
    ws = torch.empty(int(_native.lib().omb_reduce_workspace_bytes(M)) // 8 + 1, dtype=torch.float64, device=x.device)
    out = []
    for f in range(F):
        v = ctypes.c_double()
        _native.call("omb_loglik", ctypes.c_void_p(m.data_ptr() + 4 * f * M), ctypes.c_void_p(fp.data_ptr() + 4 * f * M),
                     M, float(o.epps), ctypes.byref(v), _ptr(ws), st)
        out.append(v.value)
    return np.array(out)


class Dataset:
    """x2 / x20 OSEM images of `n` seeded studies (kept on the device)."""

    def __init__(self, o, first_seed, n, counts, batch=24, keep_data=False, converged=0):
        import torch
        dev = torch.device("cuda", o._device)
        N = int(o.N[0])
        self.x2 = torch.empty((n, N), device=dev)
        self.x20 = torch.empty((n, N), device=dev)
        self.xc = torch.empty((n, N), device=dev) if converged else None
        self.m = [] if keep_data else None
        rng = np.random.default_rng(first_seed ^ 0x5EED)
        lo, hi = np.log(counts[0]), np.log(counts[1])
        self.counts = np.exp(rng.uniform(lo, hi, n))
        for s0 in range(0, n, batch):
            F = min(batch, n - s0)
            truth = phantoms(o, first_seed + s0, F, dev)
            m = simulate(o, truth, self.counts[s0:s0 + F], first_seed + s0)
            solver = rec.OSEMBatch(o, m, x0=np.ones(N, dtype=np.float32))
            solver.iterate(2, use_graph=True)
            self.x2[s0:s0 + F] = solver.x
            solver.iterate(18, use_graph=True)
            self.x20[s0:s0 + F] = solver.x
            if converged:
                solver.iterate(converged - 20, use_graph=True)
                self.xc[s0:s0 + F] = solver.x
            if keep_data:
                self.m.append(m)
            del truth, solver
        torch.cuda.synchronize(dev)


def sensitivity(o):
    import torch
    dev = torch.device("cuda", o._device)
    s = torch.empty(int(o.N[0]), device=dev)
    _native.call("omb_sensitivity", o._handle, -1, _ptr(s), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    return s


def train(o, data, minutes, batch=4, lr=2e-3, seed=0, log=None):
    """Adam on the mean squared error between the network's prediction from
    x2 and x20, for `minutes` of wall time; returns the network."""
    import torch
    dev = data.x2.device
    nx, ny, nz = int(o.Nx[0]), int(o.Ny[0]), int(o.Nz[0])
    N = nx * ny * nz
    net = UNet3D(nx, ny, nz, batch, dev, seed=seed)
    sens = sensitivity(o)
    sens_scale = 1.0 / float(sens.max())
    n = data.x2.shape[0]
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    step, hist = 0, []
    while time.perf_counter() - t0 < 60.0 * minutes:
        order = rng.permutation(n - n % batch)
        for i in range(0, len(order), batch):
            idx = torch.as_tensor(order[i:i + batch], device=dev)
            x2 = data.x2.index_select(0, idx).contiguous()
            x20 = data.x20.index_select(0, idx).contiguous()
            net.loss.zero_()
            net.forward(x2, N, sens, sens_scale)
            net.backward(x20, N)
            step += 1
            # cosine decay over the time budget
            frac = min((time.perf_counter() - t0) / (60.0 * minutes), 1.0)
            net.adam_step(lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * frac))))
            if step % 50 == 0:
                hist.append((step, float(net.loss.item())))
                if log:
                    log(f"step {step} loss {hist[-1][1]:.5f} t {time.perf_counter() - t0:.0f}s")
            if time.perf_counter() - t0 >= 60.0 * minutes:
                break
    torch.cuda.synchronize(dev)
    net.history = hist
    net.train_steps = step
    return net


def _rel(a, b):
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def evaluate(o, net_state, first_seed, n, counts, converged=100, batch=8, timing_studies=8, log=None, k_fixed=4):
    """Warm start vs plain OSEM on `n` held-out studies (seeds first_seed..).

    Untimed pass: per study the continuation count k after which the warm
    path's log-likelihood first reaches the plain 20-iteration value L20.
    Timed pass (CUDA events, one study at a time): plain = 20 iterations;
    warm = 2 iterations + network + `k_fixed` iterations + one
    log-likelihood evaluation -- the same fixed continuation for every study
    (4 = the largest k over the 200-study evaluation of the committed
    weights), so no per-study knowledge enters the timed region; each timed
    study records whether that fixed path reached L20."""
    import torch
    dev = torch.device("cuda", o._device)
    nx, ny, nz = int(o.Nx[0]), int(o.Ny[0]), int(o.Nz[0])
    N = nx * ny * nz
    M = o.measurementCount(-1)
    sens = sensitivity(o)
    sens_scale = 1.0 / float(sens.max())
    floor = 1e-3
    nets = {}
    rows = []
    for s0 in range(0, n, batch):
        F = min(batch, n - s0)
        truth = phantoms(o, first_seed + s0, F, dev)
        cnt = np.exp(np.random.default_rng(first_seed + s0).uniform(np.log(counts[0]), np.log(counts[1]), F))
        m = simulate(o, truth, cnt, first_seed + s0)
        work = torch.empty(F * M, device=dev)
        plain = rec.OSEMBatch(o, m, x0=np.ones(N, dtype=np.float32))
        plain.iterate(20, use_graph=True)
        x20 = plain.x.clone()
        L20 = loglik_frames(o, x20, m, work)
        plain.iterate(converged - 20, use_graph=True)
        xconv = plain.x.clone()
        warm = rec.OSEMBatch(o, m, x0=np.ones(N, dtype=np.float32))
        warm.iterate(2, use_graph=True)
        if F not in nets:
            nets[F] = UNet3D(nx, ny, nz, F, dev)
            nets[F].load_state_dict(net_state)
        net = nets[F]
        net.forward(warm.x, N, sens, sens_scale)
        net.predict_into(warm.x, N, floor)
        L = loglik_frames(o, warm.x, m, work)
        k = np.where(L >= L20, 0, -1)
        x_at = [None] * F
        for f in range(F):
            if k[f] == 0:
                x_at[f] = warm.x[f].clone()
        for it in range(1, 21):
            if (k >= 0).all():
                break
            warm.iterate(1, use_graph=True)
            L = loglik_frames(o, warm.x, m, work)
            for f in range(F):
                if k[f] < 0 and L[f] >= L20[f]:
                    k[f] = it
                    x_at[f] = warm.x[f].clone()
        for f in range(F):
            xa = x_at[f] if x_at[f] is not None else warm.x[f]
            rows.append({"seed": first_seed + s0 + f, "counts": float(cnt[f]), "L20": float(L20[f]),
                         "k": int(k[f]) if k[f] >= 0 else None,
                         "rel_l2_plain20_vs_converged": _rel(x20[f], xconv[f]),
                         "rel_l2_warm_vs_converged": _rel(xa, xconv[f]),
                         "rel_l2_warm_vs_plain20": _rel(xa, x20[f])})
        if log:
            log(f"eval {s0 + F}/{n}: k = {k.tolist()}")
        del plain, warm, m, truth, work
    # wall time of both paths for single studies (CUDA events, graphs)
    times = []
    timed_reached = []
    net1 = UNet3D(nx, ny, nz, 1, dev)
    net1.load_state_dict(net_state)
    work1 = torch.empty(M, device=dev)
    ws1 = torch.empty(int(_native.lib().omb_reduce_workspace_bytes(M)) // 8 + 1, dtype=torch.float64, device=dev)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for r in rows[:timing_studies]:
        seed = r["seed"]
        truth = phantoms(o, seed, 1, dev)
        m = simulate(o, truth, [r["counts"]], seed)
        a = rec.OSEMBatch(o, m, x0=np.ones(N, dtype=np.float32))
        b = rec.OSEMBatch(o, m, x0=np.ones(N, dtype=np.float32))
        a.iterate(1, use_graph=True)     # capture both graphs before timing
        b.iterate(1, use_graph=True)
        a.x.fill_(1.0)
        b.x.fill_(1.0)
        net1.forward(b.x, N, sens, sens_scale)   # warm the network's kernels
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        Lw = ctypes.c_double()
        ev[0].record()
        a.iterate(20, use_graph=True)
        ev[1].record()
        b.iterate(2, use_graph=True)
        net1.forward(b.x, N, sens, sens_scale)
        net1.predict_into(b.x, N, floor)
        b.iterate(k_fixed, use_graph=True)
        # the stop test of a real run: the log-likelihood of the result
        _native.call("omb_forward_frames", o._handle, -1, 1, _ptr(b.x), N, _ptr(work1), M, st)
        _native.call("omb_loglik", _ptr(m), _ptr(work1), M, float(o.epps), ctypes.byref(Lw), _ptr(ws1), st)
        ev[2].record()
        ev[2].synchronize()
        times.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])))
        timed_reached.append(bool(Lw.value >= r["L20"]))
    ks = [r["k"] for r in rows]
    reached = [k for k in ks if k is not None]
    summary = {
        "studies": len(rows), "reached_L20": len(reached),
        "k_median": float(np.median(reached)) if reached else None,
        "k_mean": float(np.mean(reached)) if reached else None,
        "k_max": int(max(reached)) if reached else None,
        "plain_ms_median": float(np.median([t[0] for t in times])) if times else None,
        "warm_ms_median": float(np.median([t[1] for t in times])) if times else None,
        "time_ratio_median": float(np.median([t[1] / t[0] for t in times])) if times else None,
        "timed_continuation": k_fixed,
        "timed_studies": len(times), "timed_reached_L20": int(sum(timed_reached)),
        "rel_l2_plain20_vs_converged_median": float(np.median([r["rel_l2_plain20_vs_converged"] for r in rows])),
        "rel_l2_warm_vs_converged_median": float(np.median([r["rel_l2_warm_vs_converged"] for r in rows])),
        "rel_l2_warm_vs_plain20_median": float(np.median([r["rel_l2_warm_vs_plain20"] for r in rows])),
        "converged_iterations": converged,
    }
    return summary, rows


def main():
    import torch
    p = argparse.ArgumentParser()
    p.add_argument("--train", type=int, default=5000)
    p.add_argument("--eval", type=int, default=200)
    p.add_argument("--minutes", type=float, default=5.0)
    p.add_argument("--batch", type=int, default=4)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--counts", type=float, nargs=2, default=[1e7, 1e8])
    p.add_argument("--converged", type=int, default=100)
    p.add_argument("--weights", default=None, help="skip training and evaluate these weights")
    p.add_argument("--out", default="warmstart_weights.npz")
    p.add_argument("--report", default="warmstart_report.json")
    args = p.parse_args()
    torch.cuda.set_device(0)
    o = pet_geometry()
    o.initProj()
    o.autotune(n_frames=24, repeats=1)
    log = lambda s: print(s, flush=True)  # noqa: E731
    report = {"geometry": "384 crystals x 32 rings, 256x192x63 sinograms, 128x128x63 image, 16 subsets",
              "counts": args.counts}
    if args.weights:
        state = dict(np.load(args.weights))
    else:
        t0 = time.perf_counter()
        data = Dataset(o, 1_000_000, args.train, args.counts)
        report["data_seconds"] = time.perf_counter() - t0
        log(f"training data: {args.train} studies in {report['data_seconds']:.0f} s")
        net = train(o, data, args.minutes, batch=args.batch, lr=args.lr, log=log)
        state = net.state_dict()
        np.savez(args.out, **state)
        report.update({"train_studies": args.train, "train_steps": net.train_steps, "batch": args.batch,
                       "train_minutes": args.minutes, "loss_history": net.history[-20:]})
        del data
    summary, rows = evaluate(o, state, 2_000_000, args.eval, args.counts, converged=args.converged, log=log)
    report["eval"] = summary
    report["eval_rows"] = rows
    with open(args.report, "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
