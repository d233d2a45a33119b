"""Priors of the reconstruction path (omegatomo/util/priors.py): the relative
difference prior gradient, on the device."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native


def RDP(im, Nx, Ny, Nz, gamma, beta, rType=2, epps=1e-8):
    """Gradient of the relative difference prior (util/priors.py:3-200,
    RDPKernel auxKernels.cl:664-872): a new float32 CUDA tensor
    beta * dRDP(im)/dim.  ``im`` is the column-major image as a flat float32
    CUDA tensor; ``rType`` is accepted for the reference's signature (the
    input here is always a torch tensor)."""
    import torch
    n = [int(np.ravel(v)[0]) for v in (Nx, Ny, Nz)]
    if not isinstance(im, torch.Tensor) or not im.is_cuda:
        raise TypeError('RDP takes a CUDA torch tensor')
    u = im.reshape(-1).to(torch.float32).contiguous()
    grad = torch.zeros_like(u)
    st = ctypes.c_void_p(torch.cuda.current_stream(u.device).cuda_stream)
    _native.call("omb_rdp_gradient", ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(grad.data_ptr()), n[0], n[1],
                 n[2], float(gamma), float(epps), float(beta), st)
    return grad
