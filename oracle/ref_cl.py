"""TEST INFRASTRUCTURE ONLY: the reference's own GPU kernels, run on the host.

Loads ``oracle/_ref/libref_cl_<variant>_{d,f}.so`` (built by oracle/Makefile
from OMEGA's source/opencl kernels through ``cl_host_shim.h`` and
``ref_cl_wrap.cpp``) and calls them on the arrays an addProjector()-ed
projector object holds, exactly as omegatomo/projector/projfunctions.py hands
them to the CUDA kernels: the same subset slices of ``x`` / ``z``, the same
float32 scalars (voxel grid, dScale / dSize, dL, kerroin, bmax = b + N d).

``precision="d"`` runs the kernels in FP64 with exact texture weights: the
pin of the FP64 restatements in bdd_oracle.c, interp_oracle.c and oracle.py.
``precision="f"`` runs them in FP32 with the 8-bit texture weights of the
reference's GPU path (``frac_bits=8``), to state how far the reference's own
GPU arithmetic is from the FP64 answer.

Only tests/ import this module; it needs the OMEGA sources at build time, so
tests that use it skip when oracle/_ref was not built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_libs = {}
_D = ctypes.c_double
_I = ctypes.c_int
_LL = ctypes.c_longlong
_P = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_cl_bdd_fp_d.so"))


def _lib(variant, precision):
    key = (variant, precision)
    if key not in _libs:
        path = os.path.join(REF_DIR, f"libref_cl_{variant}_{precision}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle OMEGA_REFERENCE=...)")
        L = ctypes.CDLL(path)
        if hasattr(L, "refcl_bdd_fp"):
            L.refcl_bdd_fp.argtypes = [_I, _I, _D, _D, _I, _I, _I] + [_D] * 11 + [_P, _P, _LL, _P, _I, _P]
        if hasattr(L, "refcl_bdd_bp"):
            L.refcl_bdd_bp.argtypes = [_I, _I, _D, _D, _I, _I, _I] + [_D] * 11 + [_P, _P, _LL, _P, _I, _I, _P, _P]
        if hasattr(L, "refcl_interp"):
            L.refcl_interp.argtypes = [_I, _I, _D, _D, _D, _D, _P, _D, _I, _I, _I] + [_D] * 9 + \
                [_P, _LL, _P, _LL, _I, _P, _P, _P, _I]
        if hasattr(L, "refcl_interp_ct_bp"):
            L.refcl_interp_ct_bp.argtypes = [_I, _I, _D, _D, _I, _I, _I] + [_D] * 7 + [_P, _P, _LL, _P, _I, _I, _P,
                                                                                        _P]
        if hasattr(L, "refcl_tv_gradient"):
            L.refcl_tv_gradient.argtypes = [_I, _I, _I, _P, _D, _D, _D, _P]
        if hasattr(L, "refcl_pdhg_update"):
            L.refcl_pdhg_update.argtypes = [_I, _I, _I, _P, _P, _P, _D, _D, _D, _I]
        if hasattr(L, "refcl_tv_gradient_ex"):
            L.refcl_tv_gradient_ex.argtypes = [_I, _I, _I, _P, _D, _D, _D, _D, _P, _P]
        if hasattr(L, "refcl_proxtv"):
            L.refcl_proxtv.argtypes = [_I, _I, _I, _P, _P, _P, _D, _D]
        if hasattr(L, "refcl_poisson"):
            L.refcl_poisson.argtypes = [_I, _P, _P, _D, _D, _D, _I]
        if hasattr(L, "refcl_psf"):
            L.refcl_psf.argtypes = [_I, _I, _I, _P, _P, _I, _I, _I, _P]
        if hasattr(L, "refcl_nlm"):
            L.refcl_nlm.argtypes = [_I, _I, _I, _P, _P, _I, _D, _D, _D, _D, _D, _D, _D, _D, _P, _P]
        if hasattr(L, "refcl_ggmrf"):
            L.refcl_ggmrf.argtypes = [_I, _I, _I, _P, _P, _I, _D, _D, _D, _D, _D, _P]
        if hasattr(L, "refcl_hyper"):
            L.refcl_hyper.argtypes = [_I, _I, _I, _P, _P, _I, _D, _D, _D, _P]
        if hasattr(L, "refcl_rdp"):
            L.refcl_rdp.argtypes = [_I, _I, _I, _P, _D, _D, _D, _P]
        if hasattr(L, "refcl_proxtgv"):
            L.refcl_proxtgv.argtypes = [_I, _I, _I, _P, _P, _P, _P, _P, _D, _D, _D, _D, _D]
        _libs[key] = L
    return _libs[key]


def _dp(a):
    return None if a is None else a.ctypes.data_as(_P)


def _f32(v):
    return float(np.float32(np.ravel(v)[0]))


def _frac(precision):
    return 0 if precision == "d" else 8


def _scales(o, exact):
    """The scale scalars the kernels receive.  The reference hands them over
    as float32 (coordinates.py:209-269 rounds them, projfunctions.py passes
    cp.float32); ``exact`` gives the unrounded FP64 values of the same
    formulas, which isolates the algorithm from that input rounding."""
    d = [np.float64(np.ravel(v)[0]) for v in (o.dx, o.dy, o.dz)]
    N = [int(np.ravel(v)[0]) for v in (o.Nx, o.Ny, o.Nz)]
    if not exact:
        out = {k: _f32(getattr(o, k)) for k in ("dScaleX4", "dScaleY4", "dScaleZ4")}
        if o.CT and int(o.projector_type) in (5, 15, 45, 54, 51):
            out.update({k: _f32(getattr(o, k)) for k in ("dScaleX", "dScaleY", "dScaleZ", "dSizeX", "dSizeY")})
        return out
    out = {"dScaleX4": 1.0 / (d[0] * N[0]), "dScaleY4": 1.0 / (d[1] * N[1]), "dScaleZ4": 1.0 / (d[2] * N[2]),
           "dScaleX": 1.0 / (d[0] * (N[0] + 1)), "dScaleY": 1.0 / (d[1] * (N[1] + 1)),
           "dScaleZ": 1.0 / (d[2] * (N[2] + 1)), "dSizeX": 1.0 / (d[0] * N[0]), "dSizeY": 1.0 / (d[1] * N[1])}
    return out


class RefCT:
    """Cone-beam geometry of a CT projector object (types 4 and 5)."""

    def __init__(self, o, exact_inputs=False):
        self.sc = _scales(o, exact_inputs)
        self.n_rows, self.n_cols = int(o.nRowsD), int(o.nColsD)
        self.pitch = (_f32(o.dPitchX), _f32(o.dPitchY))
        self.N = tuple(int(np.ravel(v)[0]) for v in (o.Nx, o.Ny, o.Nz))
        self.b = tuple(_f32(v) for v in (o.bx, o.by, o.bz))
        self.d = tuple(_f32(v) for v in (o.dx, o.dy, o.dz))
        self.n_meas = np.asarray(o.nMeas, dtype=np.int64).ravel()
        self.n_proj = int(o.nProjections)
        self.xyz = np.asarray(o.x, dtype=np.float32).ravel().astype(np.float64)
        self.uv = np.asarray(o.z, dtype=np.float32).ravel().astype(np.float64)
        self.o = o

    @property
    def n_img(self):
        return self.N[0] * self.N[1] * self.N[2]

    def span(self, subset):
        if subset < 0:
            return 0, self.n_proj
        return int(self.n_meas[subset]), int(self.n_meas[subset + 1] - self.n_meas[subset])

    def geom(self, subset):
        p0, n = self.span(subset)
        return (np.ascontiguousarray(self.xyz[6 * p0:6 * (p0 + n)]), np.ascontiguousarray(self.uv[2 * p0:2 * (p0 + n)]),
                n)

    # -- projector type 5 ------------------------------------------------------
    def bdd_forward(self, image, subset=-1, precision="d"):
        o = self.o
        xyz, uv, n = self.geom(subset)
        img = np.ascontiguousarray(image, dtype=np.float64).ravel()
        y = np.zeros(self.n_rows * self.n_cols * n)
        _lib("bdd_fp", precision).refcl_bdd_fp(
            self.n_rows, self.n_cols, *self.pitch, *self.N, *self.b, self.sc["dSizeX"], self.sc["dSizeY"], *self.d,
            self.sc["dScaleX"], self.sc["dScaleY"], self.sc["dScaleZ"], _dp(xyz), _dp(uv), n, _dp(img), _frac(precision),
            _dp(y))
        return y

    def bdd_backward(self, y, subset=-1, sens=False, precision="d"):
        o = self.o
        xyz, uv, n = self.geom(subset)
        yy = np.ascontiguousarray(y, dtype=np.float64).ravel()
        img = np.zeros(self.n_img)
        s = np.zeros(self.n_img) if sens else None
        _lib("bdd_bp", precision).refcl_bdd_bp(
            self.n_rows, self.n_cols, *self.pitch, *self.N, *self.b, *self.d, self.sc["dScaleX"], self.sc["dScaleY"],
            self.sc["dScaleZ"], _f32(o.dSizeXBP), _f32(o.dSizeZBP), _dp(xyz), _dp(uv), n, _dp(yy), 0 if sens else 1,
            _frac(precision), _dp(img), _dp(s))
        return (img, s) if sens else img

    # -- projector type 4 (CT) ---------------------------------------------------
    def interp_forward(self, image, subset=-1, precision="d"):
        o = self.o
        xyz, uv, n = self.geom(subset)
        img = np.ascontiguousarray(image, dtype=np.float64).ravel()
        y = np.zeros(self.n_rows * self.n_cols * n)
        bmax = [_f32(np.float64(b) + N * np.float64(d)) for b, N, d in
                zip((np.ravel(o.bx)[0], np.ravel(o.by)[0], np.ravel(o.bz)[0]), self.N,
                    (np.ravel(o.dx)[0], np.ravel(o.dy)[0], np.ravel(o.dz)[0]))]
        _lib("i4_ct_fp", precision).refcl_interp(
            self.n_rows, self.n_cols, *self.pitch, _f32(o.dL), _f32(o.global_factor), None, 0.0, *self.N, *self.b,
            *bmax, self.sc["dScaleX4"], self.sc["dScaleY4"], self.sc["dScaleZ4"], _dp(xyz), xyz.size, _dp(uv), n,
            _frac(precision), _dp(img), _dp(y), None, 1)
        return y

    def interp_backward(self, y, subset=-1, sens=False, precision="d"):
        o = self.o
        xyz, uv, n = self.geom(subset)
        yy = np.ascontiguousarray(y, dtype=np.float64).ravel()
        img = np.zeros(self.n_img)
        s = np.zeros(self.n_img) if sens else None
        _lib("i4_ct_bp", precision).refcl_interp_ct_bp(
            self.n_rows, self.n_cols, *self.pitch, *self.N, *self.b, *self.d, _f32(np.ravel(o.kerroin)[0]), _dp(xyz),
            _dp(uv), n, _dp(yy), 0 if sens else 1, _frac(precision), _dp(img), _dp(s))
        return (img, s) if sens else img


class RefPET:
    """PET sinogram geometry of a projector object (type 4, whole-sinogram
    subsets: subset types >= 8 or one subset)."""

    def __init__(self, o, exact_inputs=False):
        self.sc = _scales(o, exact_inputs)
        self.o = o
        self.n_rows, self.n_cols = int(o.Ndist), int(o.Nang)
        self.pitch = (_f32(o.dPitchX), _f32(o.dPitchY))
        self.N = tuple(int(np.ravel(v)[0]) for v in (o.Nx, o.Ny, o.Nz))
        self.b = tuple(_f32(v) for v in (o.bx, o.by, o.bz))
        self.n_meas = np.asarray(o.nMeas, dtype=np.int64).ravel()
        self.n_proj = int(o.NSinos) if int(o.subsets) == 1 else int(self.n_meas[-1])
        self.xyz = np.asarray(o.x, dtype=np.float32).ravel().astype(np.float64)
        self.uv = np.asarray(o.z, dtype=np.float32).ravel().astype(np.float64)
        self.nbins = int(o.TOF_bins_used) if o.TOF else 1
        tofc = np.asarray(o.TOFCenter, dtype=np.float64).ravel()
        self.tofc = (tofc if exact_inputs else tofc.astype(np.float32).astype(np.float64)) if o.TOF else None
        self.sigma_x = (float(o.sigma_x) if exact_inputs else _f32(o.sigma_x)) if o.TOF else 0.0
        if int(o.subsets) > 1 and int(o.subsetType) < 8:
            raise ValueError("measurement-level subsets are not wired into the host-compiled reference")

    @property
    def n_img(self):
        return self.N[0] * self.N[1] * self.N[2]

    def _variant(self, fp):
        kind = "fp" if fp else "bp"
        return f"i4_pet_{kind}_nb1" if self.nbins == 1 else f"i4_pet_{kind}_tof{self.nbins}"

    def _call(self, fp, subset, precision, img, meas, sens):
        o = self.o
        p0 = 0 if subset < 0 else int(self.n_meas[subset])
        n = self.n_proj if subset < 0 else int(self.n_meas[subset + 1] - self.n_meas[subset])
        uv = np.ascontiguousarray(self.uv[2 * p0:2 * (p0 + n)])
        bmax = [_f32(np.float64(np.ravel(b)[0]) + N * np.float64(np.ravel(d)[0])) for b, N, d in
                zip((o.bx, o.by, o.bz), self.N, (o.dx, o.dy, o.dz))]
        _lib(self._variant(fp), precision).refcl_interp(
            self.n_rows, self.n_cols, *self.pitch, _f32(o.dL), _f32(o.global_factor), _dp(self.tofc), self.sigma_x,
            *self.N, *self.b, *bmax, self.sc["dScaleX4"], self.sc["dScaleY4"], self.sc["dScaleZ4"], _dp(self.xyz),
            self.xyz.size, _dp(uv), n, _frac(precision), _dp(img), _dp(meas), _dp(sens), 0 if sens is not None else 1)
        return n

    def rays(self, subset):
        n = self.n_proj if subset < 0 else int(self.n_meas[subset + 1] - self.n_meas[subset])
        return self.n_rows * self.n_cols * n

    def interp_forward(self, image, subset=-1, precision="d"):
        img = np.ascontiguousarray(image, dtype=np.float64).ravel()
        y = np.zeros(self.rays(subset) * self.nbins)
        self._call(True, subset, precision, img, y, None)
        return y

    def interp_backward(self, y, subset=-1, sens=False, precision="d"):
        yy = np.ascontiguousarray(y, dtype=np.float64).ravel()
        img = np.zeros(self.n_img)
        s = np.zeros(self.n_img) if sens else None
        self._call(False, subset, precision, img, yy, s)
        return (img, s) if sens else img


def _scalar(v, exact):
    return float(v) if exact else float(np.float32(v))


def tv_gradient(u, shape, smooth, beta, precision="d", sigma=1.0, exact_inputs=False):
    """auxKernels.cl TVKernel (plain TV, texture reads): grad += beta * dTV(u)
    with smoothing ``smooth``; the scalars go in as float32 like the
    reference's launch unless ``exact_inputs``."""
    nx, ny, nz = shape
    uu = np.ascontiguousarray(u, dtype=np.float64).ravel()
    g = np.zeros(uu.size)
    _lib("aux", precision).refcl_tv_gradient(nx, ny, nz, _dp(uu), _scalar(sigma, exact_inputs),
                                             _scalar(smooth, exact_inputs), _scalar(beta, exact_inputs), _dp(g))
    return g


def pdhg_update(im, rhs, u, shape, tau, theta=1.0, eps=1e-5, positivity=True, precision="d", exact_inputs=False):
    """auxKernels.cl PDHGUpdate (no subsets); returns the new (im, u)."""
    nx, ny, nz = shape
    a = np.ascontiguousarray(im, dtype=np.float64).ravel().copy()
    b = np.ascontiguousarray(u, dtype=np.float64).ravel().copy()
    r = np.ascontiguousarray(rhs, dtype=np.float64).ravel()
    _lib("aux", precision).refcl_pdhg_update(nx, ny, nz, _dp(a), _dp(r), _dp(b), _scalar(eps, exact_inputs),
                                             _scalar(theta, exact_inputs), _scalar(tau, exact_inputs),
                                             int(positivity))
    return a, b


_TV_LIB = {"satv": "aux_satv", "tvw1": "aux_tvw1", "anat1": "aux_anat1", "anat2": "aux_anat2", "apls": "aux_anat3"}


def tv_gradient_variant(u, shape, variant, smooth, beta, sigma=1.0, C=0.0, S=None, precision="d",
                        exact_inputs=False):
    """TVKernel built with the variant's macro (-DSATV, -DTVW1,
    -DANATOMICAL1/2/3): grad += beta * dTV(u); S the reference image (the 9
    tensor channels for 'anat1')."""
    nx, ny, nz = shape
    uu = np.ascontiguousarray(u, dtype=np.float64).ravel()
    g = np.zeros(uu.size)
    ss = None if S is None else np.ascontiguousarray(S, dtype=np.float64).ravel()
    _lib(_TV_LIB[variant], precision).refcl_tv_gradient_ex(
        nx, ny, nz, _dp(uu), _scalar(sigma, exact_inputs), _scalar(smooth, exact_inputs), _scalar(beta, exact_inputs),
        _scalar(C, exact_inputs), _dp(ss), _dp(g))
    return g


def proxtv_step(x, q, rhs, shape, sigma2, alpha, l2=True, diff_type=0, precision="d", exact_inputs=False):
    """One proximal-TV step with the reference's kernels (ProxTVGradient,
    ProxTVq, ProxTVDivergence built with -DPROXTV, -DL2 for the L2 ball,
    -DDIFFTYPE=1 for backward differences): returns (q, rhs) updated."""
    nx, ny, nz = shape
    lib = "aux_proxtv_" + ("l2" if l2 else "max") + ("_d1" if diff_type == 1 else "")
    xx = np.ascontiguousarray(x, dtype=np.float64).ravel()
    qq = np.ascontiguousarray(q, dtype=np.float64).ravel().copy()
    rr = np.ascontiguousarray(rhs, dtype=np.float64).ravel().copy()
    _lib(lib, precision).refcl_proxtv(nx, ny, nz, _dp(xx), _dp(qq), _dp(rr), _scalar(sigma2, exact_inputs),
                                      _scalar(alpha, exact_inputs))
    return qq.reshape(3, -1), rr


def proxtgv_step(x, q, r, v, rhs, shape, sigma2, alpha0, alpha1, theta, tau, l2=True, three_d=True, precision="d",
                 exact_inputs=False):
    """One proximal TGV step with the reference's kernels (-DPROXTV -DPROXTGV,
    -DTGVZ for 3-D, -DL2 for the L2 balls): returns (q, r, v, rhs)."""
    nx, ny, nz = shape
    lib = "aux_proxtgv" + ("" if three_d else "2d") + ("_l2" if l2 else "_max")
    xx = np.ascontiguousarray(x, dtype=np.float64).ravel()
    qq = np.ascontiguousarray(q, dtype=np.float64).ravel().copy()
    rr = np.ascontiguousarray(r, dtype=np.float64).ravel().copy()
    vv = np.ascontiguousarray(v, dtype=np.float64).ravel().copy()
    hh = np.ascontiguousarray(rhs, dtype=np.float64).ravel().copy()
    e = exact_inputs
    _lib(lib, precision).refcl_proxtgv(nx, ny, nz, _dp(xx), _dp(qq), _dp(rr), _dp(vv), _dp(hh), _scalar(sigma2, e),
                                       _scalar(alpha0, e), _scalar(alpha1, e), _scalar(theta, e), _scalar(tau, e))
    return qq.reshape(3, -1), rr.reshape(6 if three_d else 3, -1), vv.reshape(3 if three_d else 2, -1), hh


def rdp_gradient(u, shape, gamma, epps, beta, images=True, precision="d", exact_inputs=False):
    """RDPKernel of the reference (-DRDP; images: the clamp-to-edge texture,
    else the buffer): beta * dRDP(u), flat, x fastest."""
    nx, ny, nz = shape
    uu = np.ascontiguousarray(u, dtype=np.float64).ravel()
    g = np.zeros(uu.size)
    e = exact_inputs
    _lib("aux_rdp" if images else "aux_rdp_buf", precision).refcl_rdp(
        nx, ny, nz, _dp(uu), _scalar(gamma, e), _scalar(epps, e), _scalar(beta, e), _dp(g))
    return g


def ggmrf_gradient(u, shape, weights, p, q, c, pqc, beta, precision="d", exact_inputs=False):
    """GGMRFKernel of the reference (-DGGMRF, 3 x 3 x 3 window): beta * dGGMRF(u)."""
    nx, ny, nz = shape
    uu = np.ascontiguousarray(u, dtype=np.float64).ravel()
    w = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    g = np.zeros(uu.size)
    e = exact_inputs
    _lib("aux_ggmrf", precision).refcl_ggmrf(nx, ny, nz, _dp(uu), _dp(w), w.size, _scalar(p, e), _scalar(q, e),
                                             _scalar(c, e), _scalar(pqc, e), _scalar(beta, e), _dp(g))
    return g


def hyperbolic_gradient(u, shape, weights, delta, beta, epps=1e-8, precision="d", exact_inputs=False):
    """hyperbolicKernel of the reference (-DHYPER, 3 x 3 x 3 window): beta * dHyperbolic(u)."""
    nx, ny, nz = shape
    uu = np.ascontiguousarray(u, dtype=np.float64).ravel()
    w = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    g = np.zeros(uu.size)
    e = exact_inputs
    _lib("aux_hyper", precision).refcl_hyper(nx, ny, nz, _dp(uu), _dp(w), w.size, _scalar(delta, e),
                                             _scalar(epps, e), _scalar(beta, e), _dp(g))
    return g


def nlm_gradient(u, shape, gaussian, h, epps, beta, variant="nlm0", gamma=10.0, ggmrf=(2.0, 1.5, 0.001),
                 adaptive_s=0.0, u_ref=None, precision="d", exact_inputs=False):
    """The reference's NLM kernel built as `variant` (aux_<variant>: nlm0, nlm1, nlm3, nlm6, nlm0ar), search
    and patch windows 3 x 3 x 3: beta * g(u)."""
    nx, ny, nz = shape
    uu = np.ascontiguousarray(u, dtype=np.float64).ravel()
    gg = np.ascontiguousarray(gaussian, dtype=np.float64).ravel()
    rr = np.ascontiguousarray(u_ref if u_ref is not None else uu, dtype=np.float64).ravel()
    g = np.zeros(uu.size)
    e = exact_inputs
    p, q, c = ggmrf
    _lib("aux_" + variant, precision).refcl_nlm(nx, ny, nz, _dp(uu), _dp(gg), gg.size, _scalar(h, e),
                                                _scalar(epps, e), _scalar(beta, e), _scalar(gamma, e),
                                                _scalar(p, e), _scalar(q, e), _scalar(c, e), _scalar(adaptive_s, e),
                                                _dp(rr), _dp(g))
    return g


def psf_convolve(x, shape, window, g, precision="d"):
    """The reference's Convolution3D_f (-DPSF): the window applied at every voxel, faces mirrored."""
    nx, ny, nz = shape
    xx = np.ascontiguousarray(x, dtype=np.float64).ravel()
    w = np.ascontiguousarray(window, dtype=np.float64).ravel()
    out = np.zeros(xx.size)
    _lib("aux_psf", precision).refcl_psf(nx, ny, nz, _dp(xx), _dp(w), int(g[0]), int(g[1]), int(g[2]), _dp(out))
    return out


def poisson_update(kind, x, rhs, lam, eps, alpha, positivity=True, precision="d", exact_inputs=False):
    """PoissonUpdate of the reference built with -DPKMA / -DMBSREM / -DBSREM: the new image."""
    xx = np.ascontiguousarray(x, dtype=np.float64).ravel().copy()
    rr = np.ascontiguousarray(rhs, dtype=np.float64).ravel()
    e = exact_inputs
    _lib("aux_" + kind.lower(), precision).refcl_poisson(xx.size, _dp(xx), _dp(rr), _scalar(lam, e), _scalar(eps, e),
                                                         _scalar(alpha, e), 1 if positivity else 0)
    return xx
