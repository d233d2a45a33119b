"""The C-ABI library loads, exports every entry point declared in
include/*.h, and rejects bad descriptors with status codes and
messages.  CPU only: no call here reaches the GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO
from omega_b200 import _native


def declared_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(REPO, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(REPO, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(omb_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _native.lib()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(L, n), n
    bound = {e[0] for e in _native.EXPORTS}
    assert set(names) <= bound, set(names) - bound


def test_abi_version_and_struct_size():
    """The library checks struct_size == sizeof(omb_geometry_desc) first; a
    descriptor that gets past that check proves the ctypes mirror's size."""
    L = _native.lib()
    assert L.omb_abi_version() == _native.OMB_ABI_VERSION
    nm = np.array([0, 2], dtype=np.int64)
    xy = np.zeros(64, dtype=np.float32)
    z = np.zeros(4, dtype=np.float32)
    d = _desc(n_meas=_native.i64_ptr(nm), xy=_native.f32_ptr(xy), n_xy=64, z=_native.f32_ptr(z), n_z=4)
    h = ctypes.c_void_p()
    st = L.omb_create(ctypes.byref(d), ctypes.byref(h))
    if st == 0:  # a GPU is present: the descriptor was accepted
        L.omb_destroy(h)
    else:
        assert "struct_size" not in L.omb_last_error().decode()


def _desc(**kw):
    d = _native.GeometryDesc()
    d.struct_size = ctypes.sizeof(_native.GeometryDesc)
    d.abi_version = _native.OMB_ABI_VERSION
    d.modality = _native.OMB_PET_SINOGRAM
    d.fp_type = d.bp_type = 1
    d.nx = d.ny = d.nz = 8
    d.dx = d.dy = d.dz = 1.0
    d.n_rows_d, d.n_cols_d = 4, 4
    d.n_proj = 2
    d.n_subsets = 1
    d.subset_type = 8
    d.tof_bins = 1
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("field,value,msg", [
    ("struct_size", 8, "struct_size"),
    ("abi_version", 99, "abi_version"),
    ("fp_type", 7, "forward projector type 7"),
    ("nx", 0, "image size"),
    ("tof_bins", 40, "TOF bin count"),
])
def test_create_rejects_bad_descriptor(field, value, msg):
    nm = np.array([0, 2], dtype=np.int64)
    xy = np.zeros(64, dtype=np.float32)
    z = np.zeros(4, dtype=np.float32)
    d = _desc(n_meas=_native.i64_ptr(nm), xy=_native.f32_ptr(xy), n_xy=64, z=_native.f32_ptr(z), n_z=4)
    setattr(d, field, value)
    h = ctypes.c_void_p()
    st = _native.lib().omb_create(ctypes.byref(d), ctypes.byref(h))
    assert st != 0 and not h.value
    assert msg in _native.lib().omb_last_error().decode()


def test_create_rejects_inconsistent_arrays():
    nm = np.array([0, 1], dtype=np.int64)  # does not reach n_proj
    xy = np.zeros(64, dtype=np.float32)
    z = np.zeros(4, dtype=np.float32)
    d = _desc(n_meas=_native.i64_ptr(nm), xy=_native.f32_ptr(xy), n_xy=64, z=_native.f32_ptr(z), n_z=4)
    h = ctypes.c_void_p()
    assert _native.lib().omb_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert "n_meas" in _native.lib().omb_last_error().decode()


def test_null_handle_calls_fail_cleanly():
    L = _native.lib()
    assert L.omb_forward(None, 0, None, None, None) == -1
    assert L.omb_backward(None, 0, None, None, None, 0, None) == -1
    assert L.omb_measurement_count(None, 0) == -1
    assert L.omb_destroy(None) == 0
    assert L.omb_pdhg_dual(None, None, None, 0, 1.0, None) == -1
    assert L.omb_pdhg_primal(None, None, None, None, None, 1.0, 1.0, 0.0, 1e-4, 1, None) == -1
    assert L.omb_pdhg_iteration(None, None, None, None, None, None, 1.0, 1.0, 1.0, 0.0, 1e-4, 1, None, None,
                                None) == -1
    t = _native.Tuning(struct_size=ctypes.sizeof(_native.Tuning))
    assert L.omb_get_tuning(None, ctypes.byref(t)) == -1
    assert L.omb_set_tuning(None, ctypes.byref(t)) == -1
    assert L.omb_autotune(None, 1, 1, ctypes.byref(t), None) == -1
