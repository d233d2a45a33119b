"""Many independent CT reconstructions projected together: ``ProjectorBatch``
takes a list of ``projectorClass`` objects (after ``addProjector()``), each a
CT geometry with projector type 1 (e.g. 2-D fan-beam slices of different
sizes), and projects all of them with one persistent launch per direction
(``omb_batch_forward`` / ``omb_batch_backward`` in include/omega_b200.h).
Images and measurements of all items are concatenated flat float32 CUDA
tensors; ``image_offsets`` / ``measurement_offsets`` (length n + 1) say where
each item starts.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from .. import _native


def fanbeam_slice(n, views, detectors=None, fov=None, sod_factor=2.0, sdd_factor=4.0, projector_type=1):
    """A 2-D fan-beam CT slice as a ``projectorClass``: n x n image over `fov`
    mm (default n * 0.5 mm), `views` angles over 360 degrees, one detector row
    of `detectors` pixels (default ceil(1.5 n)) covering the magnified FOV,
    source-origin sod_factor * fov, source-detector sdd_factor * fov."""
    from .proj import projectorClass
    o = projectorClass()
    fov = float(fov if fov is not None else 0.5 * n)
    det = int(detectors if detectors is not None else math.ceil(1.5 * n))
    sod, sdd = sod_factor * fov, sdd_factor * fov
    o.CT = True
    o.nRowsD, o.nColsD = det, 1
    o.nProjections = int(views)
    o.dPitchX = o.dPitchY = 1.2 * fov * sdd / sod / det
    o.sourceToCRot, o.sourceToDetector = sod, sdd
    o.Nx = o.Ny = int(n)
    o.Nz = 1
    o.FOVa_x = o.FOVa_y = fov
    o.axial_fov = fov / n
    o.angles = np.linspace(0, 2 * np.pi, int(views), endpoint=False).astype(np.float32)
    o.projector_type = projector_type
    o.subsets, o.subsetType = 1, 8
    o.verbose = 0
    o.SinM = np.zeros((det, 1, int(views)), dtype=np.float32)  # marks projection data (not list-mode)
    o.addProjector()
    o.SinM = np.empty(0, dtype=np.float32)
    return o


class ProjectorBatch:
    def __init__(self, items):
        import torch
        if not items:
            raise ValueError("ProjectorBatch needs at least one item")
        descs = (_native.GeometryDesc * len(items))()
        keep = []
        for i, o in enumerate(items):
            if not o.projectorAdded:
                o.addProjector()
            d, k = o._descriptor()
            descs[i] = d
            keep.append(k)
        h = ctypes.c_void_p()
        _native.call("omb_batch_create", descs, len(items), ctypes.byref(h))
        del keep
        self._handle = h
        self.n = len(items)
        self._device = torch.cuda.current_device()
        L = _native.lib()
        self.image_offsets = np.array([L.omb_batch_image_offset(h, i) for i in range(self.n + 1)], dtype=np.int64)
        self.measurement_offsets = np.array([L.omb_batch_measurement_offset(h, i) for i in range(self.n + 1)],
                                            dtype=np.int64)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None:
            try:
                _native.lib().omb_batch_destroy(h)
            except Exception:
                pass
            self._handle = None

    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self._device).cuda_stream)

    def forward(self, images, out=None):
        """y = A images for every item (concatenated)."""
        import torch
        if images.numel() != int(self.image_offsets[-1]):
            raise ValueError("images must hold every item's image")
        y = out if out is not None else torch.empty(int(self.measurement_offsets[-1]), device=images.device)
        _native.call("omb_batch_forward", self._handle, ctypes.c_void_p(images.data_ptr()),
                     ctypes.c_void_p(y.data_ptr()), self._stream())
        return y

    def backward(self, y, out=None):
        """images = A^T y for every item (concatenated)."""
        import torch
        if y.numel() != int(self.measurement_offsets[-1]):
            raise ValueError("y must hold every item's measurements")
        img = out if out is not None else torch.empty(int(self.image_offsets[-1]), device=y.device)
        _native.call("omb_batch_backward", self._handle, ctypes.c_void_p(y.data_ptr()),
                     ctypes.c_void_p(img.data_ptr()), self._stream())
        return img
