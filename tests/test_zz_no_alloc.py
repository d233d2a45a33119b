"""The allocation-free fixed-point backprojection (omb_backward_fixed64_noalloc).

It serves callers that cannot call cudaMalloc because their device memory is
owned by another allocator or fixed at start-up: everything is passed in as
device buffers and the int64 scratch is a fixed device array inside the
library.  This file is collected last on purpose (pytest orders files by
name), so a run that stops at the first failure has already run every other
test.  The GPU test passes both alone in a fresh process and after the rest.
"""
import ctypes

import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc
from omega_b200 import _native


def _device_desc(o, dev):
    """A descriptor whose geometry arrays live on the device."""
    import torch
    d, keep = o._descriptor()
    dxy = torch.as_tensor(keep["xy"], device=dev)
    dz = torch.as_tensor(keep["z"], device=dev)
    d.xy = ctypes.cast(ctypes.c_void_p(dxy.data_ptr()), ctypes.POINTER(ctypes.c_float))
    d.z = ctypes.cast(ctypes.c_void_p(dz.data_ptr()), ctypes.POINTER(ctypes.c_float))
    dev_keep = [dxy, dz, keep]
    if o.TOF:
        dt = torch.as_tensor(keep["tof"], device=dev)
        d.tof_centers = ctypes.cast(ctypes.c_void_p(dt.data_ptr()), ctypes.POINTER(ctypes.c_float))
        dev_keep.append(dt)
    d.fixed64_workspace = 0
    return d, dev_keep


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["pet_mini", "pet_tof_small"])
def test_noalloc_matches_fixed64_backprojection_twice(cuda, name):
    import torch
    o = make_options(name)
    o.use_64bit_atomics = True
    o.initProj()
    d, keep = _device_desc(o, cuda)
    n = int(o.N[0])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(21)
    L = _native.lib()
    for call, subset in enumerate((0, 1)):  # two calls in a row, the second reuses the scratch
        m = o.measurementCount(subset)
        y = torch.as_tensor(rng.uniform(0.0, 2.0, m).astype(np.float32), device=cuda)
        img = torch.full((n,), -7.0, device=cuda)
        sens = torch.full((n,), -7.0, device=cuda) if call == 0 else None
        st = L.omb_backward_fixed64_noalloc(ctypes.byref(d), subset, ctypes.c_void_p(y.data_ptr()),
                                            ctypes.c_void_p(img.data_ptr()),
                                            ctypes.c_void_p(sens.data_ptr() if sens is not None else 0), stream)
        assert st == 0, L.omb_last_error().decode()
        ref_img, ref_sens = o.backwardProject(y, subset, sens=True)
        torch.cuda.synchronize()
        # both paths run the same int64 kernel and conversion: equal bit for bit
        assert np.array_equal(img.cpu().numpy().view(np.uint32), ref_img.cpu().numpy().view(np.uint32))
        if sens is not None:
            assert np.array_equal(sens.cpu().numpy().view(np.uint32), ref_sens.cpu().numpy().view(np.uint32))
        assert orc.rel_l2(img.cpu().numpy(), orc.backward(orc.Geometry(o), y.cpu().numpy(), subset)) < 1e-5


def test_noalloc_rejects_images_above_the_limit():
    """Size check happens before any CUDA call (runs without a GPU too)."""
    o = make_options("pet_mini")
    d, keep = o._descriptor()
    d.nx = d.ny = 1024
    d.nz = 2   # 2,097,152 voxels > 1,048,576
    L = _native.lib()
    st = L.omb_backward_fixed64_noalloc(ctypes.byref(d), 0, ctypes.c_void_p(16), ctypes.c_void_p(16), None, None)
    assert st == -4
    assert "exceeds the allocation-free limit of 1048576 voxels" in L.omb_last_error().decode()
