"""Parity at the full geometry of the benchmarked workloads.

* Cone-beam CT (the default bench workload): 512 x 512 panel of 0.4 mm
  pixels, SOD 500 / SDD 1000 mm, 256^3 volume of 0.25 mm voxels -- four of
  its 360 views (0, 91, 182, 273 degrees), which is where the TMA-staged
  type-5 kernels run with their benchmark boxes and straight-line footprint
  path.  Forward and backprojection (with sensitivity), staged and unstaged,
  against the FP64 oracle (itself pinned to the reference's projectorType5
  kernels on this geometry, tests/test_refcl_pin.py).
* Dynamic PET (the batching workload): 384 crystals x 32 rings,
  256 x 192 x 63 sinograms, 128 x 128 x 63 image, 16 subsets -- two frames
  of one subset through the frame-batched entries omb_forward_frames /
  omb_backward_frames in both frame layouts, against the Siddon oracle.
Every call must leave the device error word clear.
Bar: relative L2 <= 1e-5 (FP32 kernels against FP64)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _ellipsoids(g, seed):
    """Seeded ellipsoid phantom, attenuation 0-0.02 /mm."""
    rng = np.random.default_rng(seed)
    xs = (np.arange(g.nx) + 0.5) * g.d[0] + g.b[0]
    ys = (np.arange(g.ny) + 0.5) * g.d[1] + g.b[1]
    zs = (np.arange(g.nz) + 0.5) * g.d[2] + g.b[2]
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    R = abs(g.b[0])
    img = 0.01 * ((X / (0.85 * R)) ** 2 + (Y / (0.7 * R)) ** 2 + (Z / (0.9 * R)) ** 2 < 1)
    for _ in range(6):
        c = rng.uniform(-0.4, 0.4, 3) * R
        a = rng.uniform(0.05, 0.2, 3) * R
        img = img + rng.uniform(0.002, 0.01) * (((X - c[0]) / a[0]) ** 2 + ((Y - c[1]) / a[1]) ** 2 +
                                                ((Z - c[2]) / a[2]) ** 2 < 1)
    return img.ravel(order="F")


@pytest.fixture(scope="module")
def cbct(cuda):
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), CONFIGS["ct_cfg1_4v"])
    o.addProjector()
    o.initProj()
    g = orc.Geometry(o)
    x = _ellipsoids(g, 7)
    y = np.random.default_rng(8).uniform(0.0, 2.0, g.rays(0))
    ref_fp = orc.bdd_forward(g, x, 0)
    ref_bp, ref_sens = orc.bdd_backward(g, y, 0, sens=True)
    return o, x, y, ref_fp, ref_bp, ref_sens, g


@pytest.mark.parametrize("staged", [1, 0])
@pytest.mark.parametrize("columns", [8, 16])
def test_cbct_full_geometry_forward(cuda, cbct, staged, columns):
    from omega_b200 import _native
    o, x, _, ref_fp, _, _, _ = cbct
    o.tuning = {"bdd_fp_staged": staged, "bdd_fp_columns": columns}
    y = o.forwardProject(_t(x, cuda), 0).cpu().numpy()
    assert _native.lib().omb_take_device_error() == 0
    assert orc.rel_l2(y, ref_fp) < TOL


@pytest.mark.parametrize("staged", [1, 0])
def test_cbct_full_geometry_backward(cuda, cbct, staged):
    from omega_b200 import _native
    o, _, y, _, ref_bp, ref_sens, _ = cbct
    o.tuning = {"bdd_bp_staged": staged}
    img, sens = o.backwardProject(_t(y, cuda), 0, sens=True)
    assert _native.lib().omb_take_device_error() == 0
    assert orc.rel_l2(img.cpu().numpy(), ref_bp) < TOL
    assert orc.rel_l2(sens.cpu().numpy(), ref_sens) < TOL


def test_cbct_full_geometry_ray_backward(cuda, cbct):
    """The ray-driven scatter backprojection (float atomics) at the benchmark
    geometry against the FP64 adjoint of the forward projection."""
    import ctypes

    import torch
    from omega_b200 import _native
    o, _, y, _, _, _, g = cbct
    ref = orc.bdd_backward_ray(g, y, 0)
    yd = _t(y, cuda)
    img = torch.empty(g.n_img, device=cuda)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.call("omb_backward", o._handle, 0, ctypes.c_void_p(yd.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                 None, _native.OMB_BP_RAY, st)
    assert orc.rel_l2(img.cpu().numpy(), ref) < TOL
    assert _native.lib().omb_take_device_error() == 0


@pytest.mark.parametrize("layout", [0, 1])
def test_dynamic_pet_full_geometry_frames(cuda, layout):
    import os
    import sys

    import torch
    from omega_b200 import _native
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    o = bench.dynamic_pet_options()
    o.initProj()
    o.tuning = {"siddon_frame_layout": layout}
    g = orc.Geometry(o)
    n, subset, nf = g.n_img, 0, 2
    m = o.measurementCount(subset)
    imgs = bench.dynamic_images(o, 6)[[1, 4]]
    dimgs = _t(imgs, cuda)
    ys = torch.empty((nf, m), device=cuda)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.call("omb_forward_frames", o._handle, subset, nf, ctypes.c_void_p(dimgs.data_ptr()), n,
                 ctypes.c_void_p(ys.data_ptr()), m, st)
    rng = np.random.default_rng(9)
    yin = _t(rng.uniform(0.0, 3.0, (nf, m)), cuda)
    back = torch.empty((nf, n), device=cuda)
    _native.call("omb_backward_frames", o._handle, subset, nf, ctypes.c_void_p(yin.data_ptr()), m,
                 ctypes.c_void_p(back.data_ptr()), n, st)
    torch.cuda.synchronize()
    assert _native.lib().omb_take_device_error() == 0
    for f in range(nf):
        assert orc.rel_l2(ys[f].cpu().numpy(), orc.forward(g, imgs[f], subset)) < TOL, f
        assert orc.rel_l2(back[f].cpu().numpy(), orc.backward(g, yin[f].cpu().numpy(), subset)) < TOL, f
