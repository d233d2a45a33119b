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


def neighbourhood_weights(options):
    """Distance weights 1/d of the (2Ndx+1)(2Ndy+1)(2Ndz+1) neighbourhood
    (prepass.py:634-700, the non-GGMRF branch): voxel pitch FOV/N per axis,
    offsets from +Nd down to -Nd, x fastest; the centre is inf."""
    Ndx, Ndy, Ndz = int(options.Ndx), int(options.Ndy), int(options.Ndz)
    distX = float(np.ravel(options.FOVa_x)[0]) / float(np.ravel(options.Nx)[0])
    distY = float(np.ravel(options.FOVa_y)[0]) / float(np.ravel(options.Ny)[0])
    distZ = float(np.ravel(options.axial_fov)[0]) / float(np.ravel(options.Nz)[0])
    nz1 = int(np.ravel(options.Nz)[0]) == 1
    w = np.zeros((2 * Ndx + 1) * (2 * Ndy + 1) * (2 * Ndz + 1), dtype=np.float32)
    cc = np.zeros((2 * Ndy + 1) * (2 * Ndx + 1), dtype=np.float32)
    for lt, jj in enumerate(range(Ndz, -Ndz - 1, -1)):
        for ll, kk in enumerate(range(Ndy, -Ndy - 1, -1)):
            xs = np.arange(Ndx, -Ndx - 1, -1) * distX
            ys = np.repeat(kk, Ndy * 2 + 1) * distY
            if Ndz == 0 or nz1:
                apu = np.column_stack((xs, ys))
            elif Ndz != Ndx:
                zs = np.concatenate((np.zeros(Ndx - Ndz), np.repeat(jj, Ndz * 2 + 1) * distZ, np.zeros(Ndx - Ndz)))
                apu = np.column_stack((xs, ys, zs))
            else:
                apu = np.column_stack((xs, ys, np.repeat(jj, Ndz * 2 + 1) * distZ))
            cc[(Ndy * 2 + 1) * ll:(Ndy * 2 + 1) * (ll + 1)] = np.sqrt(np.sum(apu ** 2, axis=1))
        w[(Ndx * 2 + 1) * (Ndy * 2 + 1) * lt:(Ndx * 2 + 1) * (Ndy * 2 + 1) * (lt + 1)] = cc
    with np.errstate(divide='ignore'):
        return (1.0 / w).astype(np.float32)


def normalised_weights(weights):
    """quadWeights / huberWeights (prepass.py:703-744) for computed weights:
    divided by the sum of the finite ones, the centre left out."""
    w = np.asarray(weights, dtype=np.float32)
    wn = w / np.sum(w[~np.isinf(w)])
    half = np.size(wn) // 2
    wn = np.concatenate((wn[:half], wn[half + 1:]))
    return wn[~np.isinf(wn)].astype(np.float32)


def prior_window(wq, Ndx, Ndy, Ndz):
    """The gradient window of the quadratic / Huber prior (libHeader.h:
    1147-1154): the neighbours' weights negated, the centre the absolute sum,
    x fastest; applied with mirrored edges it gives sum_k w_k (x_j - x_k)."""
    n = (2 * Ndx + 1) * (2 * Ndy + 1) * (2 * Ndz + 1)
    neg = -np.asarray(wq, dtype=np.float32)
    win = np.zeros(n, dtype=np.float32)
    win[:n // 2] = neg[:n // 2]
    win[n // 2 + 1:] = neg[n // 2:]
    win[n // 2] = np.abs(np.sum(neg, dtype=np.float32))
    return win


def nlm_gaussian(options):
    """Patch weights of the non-local priors (NLMPrepass, prepass.py:797-804):
    exp(-(x^2 + y^2 + z^2) / (2 NLM_gauss^2)) on the (2 Nlx + 1)(2 Nly + 1)
    (2 Nlz + 1) patch offsets, x fastest, float32."""
    s = float(getattr(options, 'NLM_gauss', 2.0))
    axes = [np.linspace(-n, n, 2 * n + 1, dtype=np.float32)
            for n in (int(options.Nlx), int(options.Nly), int(options.Nlz))]
    g = np.exp(-(np.add.outer(np.add.outer(axes[0] ** 2 / (2 * s ** 2), axes[1] ** 2 / (2 * s ** 2)),
                              axes[2] ** 2 / (2 * s ** 2))))
    options.gaussianNLM = g.flatten('F').astype(np.float32)
    return options.gaussianNLM


def nlm_type(options):
    """NLTYPE of the options (ProjectorClass.h:841-862)."""
    if getattr(options, 'NLM_MRP', False):
        return 2
    if getattr(options, 'NLTV', False):
        return 1
    if getattr(options, 'NLRD', False):
        return 3
    if getattr(options, 'NLLange', False):
        return 4
    if getattr(options, 'NLGGMRF', False):
        return 6
    return 0


def ggmrf_weights(options):
    """GGMRF neighbour weights (computeWeights' GGMRF branch + quadWeights,
    prepass.py:661-682, 703-730): 1 / distance over the offsets x from +Nd
    down to -Nd (outermost), then y, then z (fastest), normalised by their
    sum, the centre left out; float32.  Built for cubic neighbourhoods
    (Ndx = Ndy = Ndz) of a 3-D image, the case the reference's branch forms
    consistently."""
    nd = int(options.Ndx)
    if int(options.Ndy) != nd or int(options.Ndz) != nd:
        raise ValueError('GGMRF weights are built for Ndx = Ndy = Ndz')
    dx = np.float32(np.ravel(options.FOVa_x)[0]) / np.float32(np.ravel(options.Nx)[0])
    dy = np.float32(np.ravel(options.FOVa_y)[0]) / np.float32(np.ravel(options.Ny)[0])
    dz = np.float32(np.ravel(options.axial_fov)[0]) / np.float32(np.ravel(options.Nz)[0])
    r = np.arange(nd, -nd - 1, -1)
    ox, oy, oz = np.meshgrid(r, r, r, indexing='ij')      # z fastest in C order
    d = np.sqrt((oz * dz) ** 2 + (oy * dy) ** 2 + (ox * dx) ** 2).ravel().astype(np.float32)
    with np.errstate(divide='ignore'):
        w = (1.0 / d).astype(np.float32)
    w = w / np.sum(w[~np.isinf(w)])
    return w[~np.isinf(w)].astype(np.float32)


def weighted_mean_weights(options):
    """The weighted-mean prior's weights, x fastest, float32: options.weighted_weights
    when given, as given (Weighted_mean, priors.h:103, divides them by their
    sum for the means and uses them raw in the sums of types 4-6), else
    weightedWeights (prepass.py:754-774): sqrt(2) * FOVa_x / Nx times the
    distance weights, the centre set to weighted_center_weight, normalised to
    sum 1.  Raises when the weights sum to 0."""
    w = np.asarray(getattr(options, 'weighted_weights', np.empty(0)), dtype=np.float32).ravel(order='F')
    if w.size:
        if float(np.sum(w, dtype=np.float32)) == 0.0:
            raise ValueError('weighted_weights sum to 0')
    else:
        # float32 pitch, then FP64 (the reference's sqrt(2) is a float64 scalar) until the final cast
        dist = np.float32(np.ravel(options.FOVa_x)[0]) / np.float32(np.ravel(options.Nx)[0])
        w = np.sqrt(2.) * np.float64(dist) * neighbourhood_weights(options).astype(np.float64)
        w[np.isinf(w)] = float(getattr(options, 'weighted_center_weight', 2.))
        w = w / np.sum(w)
    return np.ascontiguousarray(w, dtype=np.float32)


def _voxel_sizes(options):
    """FOVa_x / Nx, FOVa_y / Ny, axial_fov / Nz in FP64 (the prepass's dx, dy, dz)."""
    def one(v):
        return float(np.ravel(v)[0])
    return (one(options.FOVa_x) / one(options.Nx), one(options.FOVa_y) / one(options.Ny),
            one(options.axial_fov) / one(options.Nz))


def median_filter_window(options):
    """(Ndx, Ndy, Ndz) of the L-filter / FMH, checked against the offsets grids
    computeOffsets.m lays out consistently: Ndx = Ndy = Ndz, or Ndx = Ndy = 1
    with Ndz = 0."""
    nd = (int(options.Ndx), int(options.Ndy), int(options.Ndz))
    if not ((nd[0] >= 1 and nd[0] == nd[1] == nd[2]) or nd == (1, 1, 0)):
        raise ValueError('the L-filter and FMH need Ndx = Ndy = Ndz, or Ndx = Ndy = 1 with Ndz = 0')
    return nd


# the tabulated one-dimensional L-filter weights of lfilter_weights.m for 3, 9
# and 25 window values (the first half and the centre; the rest mirrored)
_LFILTER_1D = {
    3: [0.15168, 0.69663],
    9: [-0.01899, 0.02904, 0.06965, 0.23795, 0.36469],
    25: [0.0055, 0.00335, -0.00427, -0.00101, -0.00008, 0.00065, 0.00314, 0.01064, 0.02907, 0.06499, 0.11835,
         0.17195, 0.19541],
}


def lfilter_weights(options):
    """The L-filter's weights a_L, float32, one per rank of the window:
    options.a_L when given, else lfilter_weights.m.  One-dimensional
    (oneD_weights): the tabulated sets for 3, 9 and 25 values, the Laplace
    curve 0.5 exp(x / b) on linspace(-4, 0) mirrored and normalised for 67
    values or more; the optimal weights for other counts below 67 come from
    numerical integration and are not built (give options.a_L).  Otherwise
    the distance weights: 0.5 exp(x / b), x = linspace(-1.5, 0, 3), over the
    offset's distance (the centre alpha1(end) / min(dx, dy, dz); the axis
    neighbours alpha1(2) / (d |l|); the diagonals alpha1(1) over the plane or
    space diagonal, whose 3-D form is sqrt(sqrt(dx^2 + dy^2) + dz^2) as in the
    reference), normalised to sum 1."""
    a = np.asarray(getattr(options, 'a_L', np.empty(0)), dtype=np.float32).ravel(order='F')
    ndx, ndy, ndz = median_filter_window(options)
    N = (2 * ndx + 1) * (2 * ndy + 1) * (2 * ndz + 1)
    if a.size:
        if a.size != N:
            raise ValueError('a_L must have (2 Ndx + 1)(2 Ndy + 1)(2 Ndz + 1) values')
        return np.ascontiguousarray(a)
    b = 1.0 / np.sqrt(2.0)
    if bool(getattr(options, 'oneD_weights', False)):
        if N in _LFILTER_1D:
            h = np.asarray(_LFILTER_1D[N], dtype=np.float64)
            alpha = np.concatenate([h, h[:-1][::-1]])
        elif N >= 67:
            h = 0.5 * np.exp(np.linspace(-4.0, 0.0, int(np.ceil(N / 2))) / b)
            alpha = np.concatenate([h, h[:-1][::-1]])
            alpha = alpha / np.sum(alpha)
        else:
            raise ValueError('one-dimensional L-filter weights for %d values need numerical integration; '
                             'give options.a_L' % N)
        return np.ascontiguousarray(alpha, dtype=np.float32)
    dx, dy, dz = _voxel_sizes(options)
    dxy = np.sqrt(dx ** 2 + dy ** 2)
    dxz = np.sqrt(dx ** 2 + dz ** 2)
    dyz = np.sqrt(dy ** 2 + dz ** 2)
    dxyz = np.sqrt(np.sqrt(dy ** 2 + dx ** 2) + dz ** 2)
    dmin = min(dx, dy, dz)
    alpha1 = 0.5 * np.exp(np.linspace(-1.5, 0.0, min(1, ndx) + min(1, ndy) + 1) / b)
    out = []
    for lz in range(-ndz, ndz + 1):
        for ly in range(-ndy, ndy + 1):
            for lx in range(-ndx, ndx + 1):
                if ndz == 0 or lz == 0:
                    if ly == 0 and lx != 0:
                        v = alpha1[1] / (dx * abs(lx))
                    elif ly == 0 and lx == 0:
                        v = alpha1[-1] / dmin
                    elif lx == 0:
                        v = alpha1[1] / (dy * abs(ly))
                    else:
                        v = alpha1[0] / dxy
                elif lx == 0 and ly == 0:
                    v = alpha1[1] / (dz * abs(lz))
                elif lx == 0:
                    v = alpha1[0] / dyz
                elif ly == 0:
                    v = alpha1[0] / dxz
                else:
                    v = alpha1[0] / dxyz
                out.append(v)
    alpha = np.asarray(out)
    return np.ascontiguousarray(alpha / np.sum(alpha), dtype=np.float32)


def fmh_weights(options):
    """The FMH prior's line weights, float32, (2 Ndx + 1) x lines column-major
    (the layout the reference loads): options.fmh_weights when given, else
    fmhWeights.m: kerroin = fmh_center_weight^(1/4) FOVa_x / Nx; each line's
    weights kerroin over the offset's length along the line, fmh_center_weight
    at the centre, each column normalised to sum 1.  3-D (13 lines): columns
    1-9 the lines with a z step (1, 3, 7, 9 the space diagonals; 2, 8 over the
    x-z length; 4, 6 over the y-z length; 5 the z axis), 10-13 the in-plane
    lines (10, 12 the plane diagonal, 11 x, 13 y); 2-D (Nz = 1 or Ndz = 0, 4
    lines): the in-plane set.  The kernel takes column ii for its line ii,
    as the reference does."""
    ndx, ndy, ndz = median_filter_window(options)
    nz = int(np.ravel(options.Nz)[0])
    two_d = nz == 1 or ndz == 0
    lines = 4 if two_d else 13
    rows = 2 * ndx + 1
    w = np.asarray(getattr(options, 'fmh_weights', np.empty(0)), dtype=np.float32)
    if w.size:
        if w.size != rows * lines:
            raise ValueError('fmh_weights must be (2 Ndx + 1) x %d' % lines)
        return np.ascontiguousarray(w.reshape((rows, lines), order='F') if w.ndim == 1 else w).ravel(order='F')
    dx, dy, dz = _voxel_sizes(options)
    cw = float(getattr(options, 'fmh_center_weight', 4.))
    kerroin = cw ** 0.25 * dx

    def col(n, length):
        return np.asarray([cw if i == 0 else kerroin / length(i) for i in range(n, -n - 1, -1)])
    planar = [lambda i: np.sqrt((dx * i) ** 2 + (dy * i) ** 2), lambda i: abs(dx * i),
              lambda i: np.sqrt((dx * i) ** 2 + (dy * i) ** 2), lambda i: abs(dy * i)]
    if two_d:
        W = np.stack([col(ndx, f) for f in planar], axis=1)
    else:
        zl = {1: lambda i: np.sqrt(np.sqrt((dz * i) ** 2 + (dx * i) ** 2) ** 2 + (dy * i) ** 2),
              2: lambda i: np.sqrt((dz * i) ** 2 + (dx * i) ** 2),
              4: lambda i: np.sqrt((dz * i) ** 2 + (dy * i) ** 2),
              5: lambda i: abs(dz * i)}
        zl[3] = zl[7] = zl[9] = zl[1]
        zl[8] = zl[2]
        zl[6] = zl[4]
        W = np.stack([col(ndz, zl[j]) for j in range(1, 10)] + [col(ndx, f) for f in planar], axis=1)
    W = W / np.sum(W, axis=0)
    return np.ascontiguousarray(W.astype(np.float32).ravel(order='F'))


def tv_anatomical_tensor(ref, Nx, Ny, Nz, T):
    """The weighting tensor of anatomical TV type 1 (prepass.py:509-533,
    assembleS): per voxel B = I - (1 - gamma) nu nu^T, nu the unit vector of
    the reference image's negated forward differences (ordered y, x, z as the
    reference stacks them, zero past the last voxel), gamma = exp(-|d|^2 /
    T^2), B = I where the differences vanish.  Returns the 9 channels
    B[r, c] (channel 3 r + c), each an image with x fastest, concatenated:
    float32, 9 Nx Ny Nz values, as options.s holds them (prepass.py:570-580)."""
    a = np.asarray(ref, dtype=np.float32).reshape((Nx, Ny, Nz), order='F')
    dy = np.zeros_like(a)
    dx = np.zeros_like(a)
    dz = np.zeros_like(a)
    dy[:, :-1, :] = a[:, :-1, :] - a[:, 1:, :]
    dx[:-1, :, :] = a[:-1, :, :] - a[1:, :, :]
    dz[:, :, :-1] = a[:, :, :-1] - a[:, :, 1:]
    d = [v.ravel(order='F') for v in (dy, dx, dz)]
    norm = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    gamma = np.exp(-(norm * norm) / np.float32(T * T))
    nz = norm > 0
    safe = np.where(nz, norm, np.float32(1.0))
    nu = [np.where(nz, v / safe, np.float32(0.0)) for v in d]
    one_minus = np.float32(1.0) - gamma
    out = np.empty((9, norm.size), dtype=np.float32)
    for r in range(3):
        for c in range(3):
            # float32 (1 - gamma) (nu_r nu_c), subtracted from the identity in FP64
            prod = np.where(nz, one_minus * (nu[r] * nu[c]), np.float32(0.0))
            out[3 * r + c] = float(r == c) - prod.astype(np.float64)
    return out.ravel()


def _reference_image(img, n, what, normalise):
    r = np.asarray(img, dtype=np.float32)
    if r.size != n:
        raise ValueError(what + ' must have the size of the image (Nx * Ny * Nz values)')
    r = r.ravel(order='F') if r.ndim > 1 else r.ravel()
    if normalise:
        # min-max normalised to [0, 1] in float32 (prepass.py:564-566)
        r = r - np.min(r)
        top = np.max(r)
        if not top > 0:
            raise ValueError(what + ' is constant')
        r = r / top
    return np.ascontiguousarray(r, dtype=np.float32)


def tv_setup(options, apls=False):
    """The TV gradient the reference builds for the TV options (ProjectorClass.h:
    900-918 kernel choice, functions.hpp:1096-1113 scalars, libHeader.h:1108-
    1124 and 1232-1245 option reads): returns (variant, sigma, C, smoothing,
    reference array or None) with variant an omb_tv_variant.

    Without TV_use_anatomical: TVtype 4 is SATV and 6 the weighted TV, both
    with sigma = SATVPhi; other types are the plain TV.  With it, the
    reference image TV_referenceImage is min-max normalised and TVtype 1
    weights the differences with the tensor of tv_anatomical_tensor (options.T),
    TVtype 2 adds C |grad ref|^2 (options.C), TVtype 5 is APLS with C =
    options.eta; other types are the plain TV.  options.APLS (apls=True) is
    APLS with the unnormalised APLS_ref_image, C = eta and the smoothing
    APLSsmoothing.  Reference images are arrays of Nx * Ny * Nz values (the
    reference's file loading and resizing are not part of this path)."""
    Nx, Ny, Nz = (int(np.ravel(getattr(options, k))[0]) for k in ('Nx', 'Ny', 'Nz'))
    n = Nx * Ny * Nz
    smooth = float(getattr(options, 'TVsmoothing', 1e-2))
    if apls:
        ref = _reference_image(options.APLS_ref_image, n, 'APLS_ref_image', False)
        return (_native.OMB_TV_APLS, 0.0, float(getattr(options, 'eta', 1e-5)),
                float(getattr(options, 'APLSsmoothing', 1e-5)), ref)
    tvtype = int(getattr(options, 'TVtype', 1))
    if not getattr(options, 'TV_use_anatomical', False):
        phi = float(getattr(options, 'SATVPhi', 1.0))
        if tvtype == 4:
            return _native.OMB_TV_SATV, phi, 0.0, smooth, None
        if tvtype == 6:
            return _native.OMB_TV_W1, phi, 0.0, smooth, None
        return _native.OMB_TV_PLAIN, 0.0, 0.0, smooth, None
    if tvtype not in (1, 2, 5):
        return _native.OMB_TV_PLAIN, 0.0, 0.0, smooth, None
    ref = _reference_image(options.TV_referenceImage, n, 'TV_referenceImage', True)
    if tvtype == 1:
        if getattr(options, 'T', None) is None:
            raise ValueError('anatomical TV type 1 needs options.T')
        return _native.OMB_TV_ANAT1, 0.0, 0.0, smooth, tv_anatomical_tensor(ref, Nx, Ny, Nz, float(options.T))
    if tvtype == 2:
        return _native.OMB_TV_ANAT2, 0.0, float(getattr(options, 'C', 1.0)), smooth, ref
    return _native.OMB_TV_APLS, 0.0, float(getattr(options, 'eta', 1e-5)), smooth, ref
