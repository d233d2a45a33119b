"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the projector path.

Loads ``oracle/liboracle.so`` (the FP64 restatement in siddon_oracle.c) and,
when built, ``oracle/_ref/libref_siddon.so`` (the reference's own OpenMP CPU
projector, projector_functions.h:1312), and restates the OSEM loop in numpy.
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module; the product never does.

OSEM restatement (the reference's compiled loop, CS-2):
  fp = A_s x + epps                      computeForwardProject.h:20-21
  r  = y_s / fp, NaN/Inf -> epps          computeForwardProject.h:92-95, 400-401
  rhs = A_s^T r
  sens_s = max(A_s^T 1, epps)             reconstructionAF.h:303-328, functions.hpp:2980-2996
  x = x / sens_s * (rhs + epps)           algorithms.h:12-15, subiterStep.h:118-121
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_siddon.so")


class OracleCT(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("bx", ctypes.c_double), ("by", ctypes.c_double), ("bz", ctypes.c_double),
        ("n_rows", ctypes.c_int), ("n_cols", ctypes.c_int),
        ("proj0", ctypes.c_int64), ("n_proj", ctypes.c_int64),
        ("pitch_x", ctypes.c_double), ("pitch_y", ctypes.c_double),
        ("xy", ctypes.POINTER(ctypes.c_float)),
        ("uv", ctypes.POINTER(ctypes.c_float)),
    ]


class OracleGeom(ctypes.Structure):
    _fields_ = [
        ("modality", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("bx", ctypes.c_double), ("by", ctypes.c_double), ("bz", ctypes.c_double),
        ("n_rows", ctypes.c_int), ("n_cols", ctypes.c_int),
        ("proj0", ctypes.c_int64), ("n_proj", ctypes.c_int64), ("m_size", ctypes.c_int64),
        ("stype", ctypes.c_int), ("n_subsets", ctypes.c_int), ("cur_subset", ctypes.c_int),
        ("pitch_x", ctypes.c_double), ("pitch_y", ctypes.c_double),
        ("global_factor", ctypes.c_double), ("epps", ctypes.c_double),
        ("nbins", ctypes.c_int),
        ("sigma_x", ctypes.c_double),
        ("tof_centers", ctypes.POINTER(ctypes.c_double)),
        ("xy", ctypes.POINTER(ctypes.c_float)),
        ("z", ctypes.POINTER(ctypes.c_float)),
        ("w", ctypes.POINTER(ctypes.c_double)),
        ("mu", ctypes.POINTER(ctypes.c_double)),
        ("tr", ctypes.POINTER(ctypes.c_uint16)),
        ("ax", ctypes.POINTER(ctypes.c_uint16)),
        ("nr_xy", ctypes.c_int), ("nr_z", ctypes.c_int),
        ("cr_xy", ctypes.c_double), ("cr_z", ctypes.c_double),
        ("proj_type", ctypes.c_int), ("orth_width", ctypes.c_double),
        ("crystxy", ctypes.c_int), ("crystz", ctypes.c_int),
        ("bmin", ctypes.c_double), ("bmax", ctypes.c_double), ("vmax", ctypes.c_double),
        ("V", ctypes.POINTER(ctypes.c_double)), ("nv", ctypes.c_int),
        ("cpu_mode", ctypes.c_int),
    ]


_lib = None
_ref = None


def build():
    """Builds the oracle libraries (oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.POINTER(ctypes.c_double)
        G = ctypes.POINTER(OracleGeom)
        L.oracle_siddon_fp.argtypes = [G, P, P]
        L.oracle_siddon_bp.argtypes = [G, P, P, P]
        L.oracle_siddon_count.argtypes = [G]
        L.oracle_siddon_count.restype = ctypes.c_int64
        C = ctypes.POINTER(OracleCT)
        L.oracle_bdd_fp.argtypes = [C, P, P]
        L.oracle_bdd_bp.argtypes = [C, P, P, P]
        L.oracle_bdd_bp_ray.argtypes = [C, P, P, P]
        L.oracle_orth_fp.argtypes = [G, P, P]
        L.oracle_orth_bp.argtypes = [G, P, P, P]
        L.oracle_interp_fp.argtypes = [G, ctypes.c_double, P, P]
        L.oracle_interp_bp.argtypes = [G, ctypes.c_double, P, P, P]
        L.oracle_interp_ct_bp.argtypes = [C, ctypes.c_double, P, P, P]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own CPU projector, or None when it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        L = ctypes.CDLL(REF_LIB)
        for name, T in (("ref_siddon_d", ctypes.c_double), ("ref_siddon_f", ctypes.c_float)):
            P = ctypes.POINTER(T)
            u = ctypes.c_uint32
            getattr(L, name).argtypes = [ctypes.c_int, u, u, u, T, T, T, T, T, T, u, u, u, P, P, P, P, P, u, T, P, T,
                                         T, u]
        P = ctypes.POINTER(ctypes.c_double)
        L.ref_listmode_d.argtypes = [ctypes.c_int, u, u, u] + [ctypes.c_double] * 6 + [ctypes.c_int64, P, P, P, P,
                                                                                      ctypes.c_double, ctypes.c_double, u]
        L.ref_multiray_d.argtypes = [ctypes.c_int, u, u, u] + [ctypes.c_double] * 6 + [u, u, u] + [P] * 5 + \
            [u, ctypes.c_double, P, ctypes.c_double, ctypes.c_double, u, u, u, ctypes.c_double, ctypes.c_double]
        L.ref_siddon_corr_d.argtypes = [ctypes.c_int, u, u, u] + [ctypes.c_double] * 6 + [u, u, u] + [P] * 5 + \
            [u, ctypes.c_double, P, ctypes.c_double, ctypes.c_double, u, P, P, ctypes.c_int, P]
        L.ref_orth_d.argtypes = [ctypes.c_int, u, u, u] + [ctypes.c_double] * 6 + [u, u, u] + [P] * 5 + \
            [u, ctypes.c_double, P, ctypes.c_double, ctypes.c_double, u, ctypes.c_int, ctypes.c_double, P, P, P,
             ctypes.c_double, ctypes.c_double, ctypes.c_double, P, P, P]
        _ref = L
    return _ref


class Geometry:
    """Everything the oracle needs from an addProjector()-ed options object."""

    def __init__(self, o):
        self.ct = bool(o.CT)
        # 0 sinogram, 1 CT, 2 list-mode events, 3 index-based events
        self.modality = 1 if self.ct else (0 if not getattr(o, 'listmode', 0) else
                                           (3 if o.useIndexBasedReconstruction else 2))
        if self.modality == 3:
            self.tr = np.ascontiguousarray(np.asarray(o.trIndex, dtype=np.uint16).ravel())
            self.ax = np.ascontiguousarray(np.asarray(o.axIndex, dtype=np.uint16).ravel())
        self.nx, self.ny, self.nz = (int(np.asarray(v).ravel()[0]) for v in (o.Nx, o.Ny, o.Nz))
        self.d = tuple(float(np.asarray(v).ravel()[0]) for v in (o.dx, o.dy, o.dz))
        self.b = tuple(float(np.asarray(v).ravel()[0]) for v in (o.bx, o.by, o.bz))
        self.n_rows, self.n_cols = int(o.nRowsD), int(o.nColsD)
        self.n_proj = int(o.nProjections)
        self.n_subsets = int(o.subsets)
        self.stype = int(o.subsetType)
        self.n_meas = np.asarray(o.nMeas, dtype=np.int64).ravel()
        self.xy = np.ascontiguousarray(np.asarray(o.x, dtype=np.float32).ravel())
        self.z = np.ascontiguousarray(np.asarray(o.z, dtype=np.float32).ravel())
        # CT: the detector pitch as the kernels receive it, a float32 scalar
        # (projfunctions.py passes cp.float32(dPitchX / dPitchY))
        self.pitch = (float(np.float32(o.dPitchX)), float(np.float32(o.dPitchY))) if self.ct else \
            (float(o.dPitchX), float(o.dPitchY))
        self.global_factor = float(o.global_factor)
        self.epps = float(o.epps)
        self.nbins = int(o.TOF_bins_used) if o.TOF else 1
        self.sigma_x = float(o.sigma_x)
        self.tofc = np.ascontiguousarray(np.asarray(o.TOFCenter, dtype=np.float64).ravel()) if o.TOF else \
            np.zeros(1, dtype=np.float64)
        # projector type 4: sampling length and the CT backprojection weight
        # the sampling length as the kernels receive it, a float32 scalar
        self.dL = float(np.float32(o.dL))
        self.kerroin = float(np.ravel(o.kerroin)[0]) if np.size(o.kerroin) else 0.0
        # PET multi-ray: rays per LOR over the crystal pitches (dPitchX
        # transaxially, dPitchY axially, as the reference's kernels take them)
        self.nr_xy = 1 if self.ct else int(getattr(o, 'n_rays_transaxial', 1))
        self.nr_z = 1 if self.ct else int(getattr(o, 'n_rays_axial', 1))
        # PET corrections: weight per measurement of all subsets (subset
        # order) and attenuation image, FP64; None when off
        self.w = None
        self.mu = None
        # projector types 2 / 3: the forward / backward type, the tube and the type-3 table
        fb = o._fp_bp_types() if hasattr(o, '_fp_bp_types') and not self.ct else (1, 1)
        self.fp_type, self.bp_type = fb
        self.tube_width = float(getattr(o, 'tube_width_z', 0.0))
        self.tube_radius = float(getattr(o, 'tube_radius', 1.0))
        self.crystxy = int(bool(getattr(o, 'orthTransaxial', False)))
        self.crystz = int(bool(getattr(o, 'orthAxial', False)))
        self.V = np.ascontiguousarray(np.asarray(getattr(o, 'V', np.zeros(1)), dtype=np.float64).ravel())
        self.vol = tuple(float(getattr(o, k, 0.0)) for k in ('bmin', 'bmax', 'Vmax'))
        self.cpu_mode = 0

    @property
    def n_img(self):
        return self.nx * self.ny * self.nz

    def meas_level(self):
        # list-mode events come in subset order: contiguous, like whole sinograms
        return self.n_subsets > 1 and self.stype < 8 and self.modality == 0

    def rays(self, subset):
        nbin = self.n_rows * self.n_cols
        if self.meas_level():
            return int(self.n_meas[subset + 1] - self.n_meas[subset])
        if subset < 0:
            return self.n_proj * nbin
        return int(self.n_meas[subset + 1] - self.n_meas[subset]) * nbin

    def struct(self, subset):
        g = OracleGeom()
        g.modality = self.modality
        g.nx, g.ny, g.nz = self.nx, self.ny, self.nz
        g.dx, g.dy, g.dz = self.d
        g.bx, g.by, g.bz = self.b
        g.n_rows, g.n_cols = self.n_rows, self.n_cols
        if self.meas_level():
            g.stype = self.stype
            g.proj0 = 0
            g.n_proj = self.n_proj
        else:
            g.stype = 0
            g.proj0 = 0 if subset < 0 else int(self.n_meas[subset])
            g.n_proj = self.n_proj if subset < 0 else int(self.n_meas[subset + 1] - self.n_meas[subset])
        g.m_size = self.rays(subset)
        g.n_subsets = self.n_subsets
        g.cur_subset = max(subset, 0)
        g.pitch_x, g.pitch_y = self.pitch
        g.global_factor = self.global_factor
        g.epps = self.epps
        g.nbins = self.nbins
        g.sigma_x = self.sigma_x
        g.tof_centers = self.tofc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.xy = self.xy.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        g.z = self.z.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        P = ctypes.POINTER(ctypes.c_double)
        if self.w is not None:
            w0 = int(self.n_meas[max(subset, 0)]) if self.meas_level() else \
                (0 if subset < 0 else int(self.n_meas[subset]) * self.n_rows * self.n_cols)
            self._w = np.ascontiguousarray(self.w, dtype=np.float64).ravel()[w0:w0 + g.m_size]
            g.w = self._w.ctypes.data_as(P)
        if self.mu is not None:
            self._mu = np.ascontiguousarray(self.mu, dtype=np.float64).ravel()
            g.mu = self._mu.ctypes.data_as(P)
        g.nr_xy, g.nr_z = self.nr_xy, self.nr_z
        g.cr_xy, g.cr_z = self.pitch
        if self.modality == 3:
            U = ctypes.POINTER(ctypes.c_uint16)
            g.tr = self.tr.ctypes.data_as(U)
            g.ax = self.ax.ctypes.data_as(U)
        g.crystxy, g.crystz = self.crystxy, self.crystz
        g.bmin, g.bmax, g.vmax = self.vol
        g.V = self.V.ctypes.data_as(P)
        g.nv = self.V.size
        g.cpu_mode = self.cpu_mode
        return g

    def orth_struct(self, subset, proj_type):
        g = self.struct(subset)
        g.proj_type = proj_type
        g.orth_width = self.tube_width if proj_type == 2 else self.tube_radius
        return g


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def forward(geom: Geometry, image, subset):
    """FP64 y = A_s image (all TOF bins, [bin0 rays, bin1 rays, ...])."""
    img = np.ascontiguousarray(image, dtype=np.float64).ravel()
    g = geom.struct(subset)
    y = np.zeros(g.m_size * geom.nbins, dtype=np.float64)
    lib().oracle_siddon_fp(ctypes.byref(g), _dp(img), _dp(y))
    return y


def backward(geom: Geometry, y, subset, sens=False):
    """FP64 A_s^T y (and A_s^T 1 when sens).  y may be None (sensitivity only)."""
    g = geom.struct(subset)
    yy = None if y is None else np.ascontiguousarray(y, dtype=np.float64).ravel()
    img = np.zeros(geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    lib().oracle_siddon_bp(ctypes.byref(g), _dp(yy), _dp(img), _dp(s))
    return (img, s) if sens else img


def orth_forward(geom: Geometry, image, subset):
    """FP64 y = A_s image with the forward projector type 2 or 3 of geom."""
    img = np.ascontiguousarray(image, dtype=np.float64).ravel()
    g = geom.orth_struct(subset, geom.fp_type)
    y = np.zeros(g.m_size * geom.nbins, dtype=np.float64)
    if lib().oracle_orth_fp(ctypes.byref(g), _dp(img), _dp(y)) != 0:
        raise ValueError("oracle_orth_fp: projector type must be 2 or 3")
    return y


def orth_backward(geom: Geometry, y, subset, sens=False):
    """FP64 A_s^T y (and A_s^T 1 when sens) with the backprojector type 2 or 3 of geom."""
    g = geom.orth_struct(subset, geom.bp_type)
    yy = None if y is None else np.ascontiguousarray(y, dtype=np.float64).ravel()
    img = np.zeros(geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    if lib().oracle_orth_bp(ctypes.byref(g), _dp(yy), _dp(img), _dp(s)) != 0:
        raise ValueError("oracle_orth_bp: projector type must be 2 or 3")
    return (img, s) if sens else img


def intersections(geom: Geometry, subset):
    """Total voxel-intersection count sum_rays Np of one call."""
    g = geom.struct(subset)
    return int(lib().oracle_siddon_count(ctypes.byref(g)))


def osem(geom: Geometry, y_subsets, x0, n_iter, forward=None, backward=None, randoms=None, prior_grad=None):
    """Restated OSEM loop in FP64; returns the image after n_iter iterations.
    The projector pair defaults to the Siddon restatement (type 1).
    randoms: per subset, added to the forward projection before the ratio
    (computeForwardProject.h:46-71), tiled over TOF bins.  prior_grad(x):
    one-step-late OSEM with that prior gradient (weight included)."""
    fwd = forward or globals()["forward"]
    bwd = backward or globals()["backward"]
    x = np.asarray(x0, dtype=np.float64).copy()
    eps = geom.epps
    sens = []
    for s in range(geom.n_subsets):
        _, sv = bwd(geom, None, s, sens=True)
        sens.append(np.maximum(sv, eps))
    for _ in range(n_iter):
        for s in range(geom.n_subsets):
            fp = fwd(geom, x, s) + eps
            if randoms is not None:
                fp = fp + np.tile(np.asarray(randoms[s], dtype=np.float64), geom.nbins)
            with np.errstate(divide="ignore", invalid="ignore"):
                r = np.asarray(y_subsets[s], dtype=np.float64) / fp
            r[~np.isfinite(r)] = eps
            if prior_grad is not None:
                # one-step-late (subiterStep.h:219-226): dU of the current image
                du = prior_grad(x)
                rhs = bwd(geom, r, s)
                x = x / (sens[s] + du) * rhs
                continue
            rhs = bwd(geom, r, s)
            x = x / sens[s] * (rhs + eps)
    return x


def default_relaxation(n_iter):
    """lam[iter] = 1 / (iter / 20 + 1) in float32 (prepass.py:962-972)."""
    return np.array([1. / (i / 20. + 1.) for i in range(n_iter)], dtype=np.float32)


def default_momentum(n_iter, n_subsets, rho=0.45, delta=100.0):
    """PKMA alpha[k] = 1 + rho k / (k + delta), k the sub-iteration count, float32 (prepass.py:998-1006)."""
    k = np.arange(n_iter * n_subsets, dtype=np.float64)
    return (1.0 + (rho * k) / (k + delta)).astype(np.float32)


def precond_image(geom: Geometry, backward=None):
    """D of the PKMA / MBSREM image preconditioners (reconstructionAF.h:779-816):
    the subsets' summed A^T 1 over the subset count, zeros set to 1."""
    bwd = backward or globals()["backward"]
    d = sum(bwd(geom, None, s, sens=True)[1] for s in range(geom.n_subsets))
    if geom.n_subsets > 1:
        d = d / geom.n_subsets
    return np.where(d == 0.0, 1.0, d)


def _grad_precond(xp, shape, diff_type, v1, v2):
    """gradientPreconditioner (functions.hpp:2016-2054): f = max(1e-5,
    |grad xp| / mean(xp)), gradF = min(v2, max(v1, mean(f) / f));
    computeGradient's forward (0), backward (1) or central (2) differences."""
    X = np.asarray(xp, dtype=np.float64).reshape(shape, order='F')
    comps = []
    for a in range(3):
        Xa = np.moveaxis(X, a, 0)
        d = np.empty_like(Xa)
        if diff_type == 0:
            d[:-1] = Xa[1:] - Xa[:-1]
            d[-1] = -Xa[-1]
        elif diff_type == 1:
            d[1:] = Xa[:-1] - Xa[1:]
            d[0] = -Xa[0]
        else:
            d[1:-1] = (Xa[2:] - Xa[:-2]) * 0.5
            d[0] = Xa[1] - Xa[0]
            d[-1] = Xa[-1] - Xa[-2]
        comps.append(np.moveaxis(d, 0, a))
    f = np.maximum(1e-5, np.sqrt(comps[0] ** 2 + comps[1] ** 2 + comps[2] ** 2) / X.mean())
    f = f.mean() / f
    return np.minimum(v2, np.maximum(v1, f)).ravel(order='F')


def poisson_update(kind, x, rhs, lam, eps, alpha, positivity=True):
    """The image step after the backprojection (PoissonUpdate, auxKernels.cl:1994-2026): PKMA x_a = x - lam
    rhs, x = (1 - alpha) x + alpha max(eps, x_a); MBSREM (MRAMLA too) x + lam rhs, max(eps, .), values >= alpha
    (the bound U) set to alpha - eps; BSREM (RAMLA too) x + lam rhs x, max(eps, .)."""
    x = np.asarray(x, dtype=np.float64)
    if kind == "PKMA":
        xa = x - lam * rhs
    elif kind == "MBSREM":
        xa = x + lam * rhs
    else:
        xa = x + lam * rhs * x
    if positivity:
        xa = np.maximum(eps, xa)
    if kind == "PKMA":
        return (1.0 - alpha) * x + alpha * xa
    if kind == "MBSREM":
        return np.where(xa >= alpha, alpha - eps, xa)
    return xa


def relaxed(geom: Geometry, y_subsets, x0, n_iter, kind, lam=None, forward=None, backward=None, randoms=None,
            prior_grad=None, positivity=True, alpha=None, upper=10000.0, precond=0, ref=None, alpha_precond=None,
            grad_precond=None, curv_precond=False, meas_precond=False, auto_relax=False, relax_scaling=False,
            img_filter=None, lam_filtered=None):
    """Restated relaxed loops in FP64 (kind: "ROSEM", "RAMLA", "BSREM",
    "ROSEM_MAP", "PKMA", "MRAMLA", "MBSREM"); returns the image after n_iter
    iterations.
    ROSEM sub-iteration (algorithms.h:102-106): x + lam x / sens (rhs - sens),
    rhs the backprojection of y / (fp + epps [+ r]).
    RAMLA / BSREM (computeForwardProject.h:98-122, auxKernels.cl:1997-2026):
    x + lam rhs x, rhs the backprojection of y / (fp + epps [+ r]) - 1, then
    max(epps, x) with positivity.  BSREM / ROSEM-MAP end each iteration with
    the MAP step x - lam x dU, x < epps -> epps (iterStep.h:14-34,
    algorithms.h:130-135); dU = prior_grad(x), weight included.
    PKMA (computeForwardProject.h:126-150, algorithms.h:151-212,
    auxKernels.cl:2008-2018): g = A^T (1 - y / (fp + epps [+ r])) [+ dU at the
    sub-iteration's image]; xa = x - lam g, max(epps, xa) with positivity;
    x = (1 - a) x + a xa, a = alpha[iter * S + subset].
    MRAMLA / MBSREM (computeForwardProject.h:153-180, algorithms.h:31-52,
    auxKernels.cl:2011-2022): x + lam (A^T (y / (fp + epps [+ r]) - 1)
    [+ dU]), max(epps, .) with positivity, values >= U set to U - epps.
    precond (PKMA / MRAMLA / MBSREM, functions.hpp:2057-2106): 1 divides the
    gradient by D, 2 multiplies it by x / D (MBSREM: U - x where x >= U / 2),
    3 by max(x, max(1e-5, ref)) / D.  Before it the gradient is multiplied by
    the type-4 image (grad_precond = dict(v1, v2, init, last, diff_type):
    recomputed from the (folded) image in sub-iterations init..last, applied
    from init on) and by alpha_precond[k] (type 3); after it by the type-6
    image dP = sum_s S / A_s^T (A_s 1 / y_s) (curv_precond).  meas_precond
    divides the ratio by A_s 1 (zeros -> 1).  PKMA with auto_relax: lam[0] =
    ||x|| / ||g|| / 4 at the first sub-iteration, lam[it] = lam[it - 1] /
    (it / 35 + 1) at each later iteration's first; relax_scaling: q = ||x|| /
    (lam ||g||), lam *= q / 1.5 when 0 < q < 1.5 (algorithms.h:151-197).
    img_filter = dict(nf, F, K): the filtering-based image preconditioner last
    (functions.hpp:2093-2099, image_filter_fft) in sub-iterations kk < K
    (K = 0: kk = 0 only, subiterStep.h:28-45); lam_filtered: the relaxation
    until sub-iteration K (never switched for K = 0), lam from K on."""
    fwd = forward or globals()["forward"]
    bwd = backward or globals()["backward"]
    lam = np.asarray(default_relaxation(n_iter) if lam is None else lam, dtype=np.float32)
    S = geom.n_subsets
    if kind == "PKMA" and alpha is None:
        alpha = default_momentum(n_iter, S)
    ramla = kind in ("RAMLA", "BSREM")
    mapstep = kind in ("BSREM", "ROSEM_MAP")
    additive = kind in ("PKMA", "MRAMLA", "MBSREM")
    x = np.asarray(x0, dtype=np.float64).copy()
    eps = geom.epps
    D = precond_image(geom, bwd) if precond else None
    shape = (geom.nx, geom.ny, geom.nz)
    lam = np.asarray(lam, dtype=np.float64).copy()
    ones = np.ones(geom.n_img)
    M = None
    if meas_precond:
        M = []
        for s in range(S):
            mv = fwd(geom, ones, s)
            mv[mv == 0] = 1.0
            M.append(mv)
    dP = None
    if curv_precond:
        dP = np.zeros(geom.n_img)
        for s in range(S):
            E = fwd(geom, ones, s)
            ys = np.asarray(y_subsets[s], dtype=np.float64)
            EE = np.where(ys > 0, E / np.where(ys > 0, ys, 1.0), 0.0)
            with np.errstate(divide="ignore", invalid="ignore"):
                dP = dP + S / bwd(geom, EE, s)
        dP[~np.isfinite(dP)] = 1.0
    gradF = None
    sens = []
    if kind in ("ROSEM", "ROSEM_MAP"):
        for s in range(S):
            _, sv = bwd(geom, None, s, sens=True)
            sens.append(np.maximum(sv, eps))
    for it in range(n_iter):
        for s in range(S):
            lm = float(lam[it])
            if img_filter is not None and lam_filtered is not None and \
                    not (img_filter["K"] > 0 and it * S + s >= img_filter["K"]):
                lm = float(lam_filtered[it])
            du = prior_grad(x) if additive and prior_grad is not None else None
            fp = fwd(geom, x, s) + eps
            if randoms is not None:
                fp = fp + np.tile(np.asarray(randoms[s], dtype=np.float64), geom.nbins)
            with np.errstate(divide="ignore", invalid="ignore"):
                r = np.asarray(y_subsets[s], dtype=np.float64) / fp
            if kind == "PKMA":
                r = 1.0 - r
            elif ramla or kind in ("MRAMLA", "MBSREM"):
                r = r - 1.0
            r[~np.isfinite(r)] = eps
            if M is not None:
                r = r / M[s]
            rhs = bwd(geom, r, s)
            if du is not None:
                rhs = rhs + du
            xp = np.where(x >= upper / 2.0, upper - x, x) if kind in ("MRAMLA", "MBSREM") else x
            kk = it * S + s
            if grad_precond is not None and kk >= grad_precond["init"]:
                if kk <= grad_precond["last"]:
                    gradF = _grad_precond(xp, shape, grad_precond.get("diff_type", 0), grad_precond["v1"],
                                          grad_precond["v2"])
                rhs = rhs * gradF
            if alpha_precond is not None:
                rhs = rhs * float(alpha_precond[kk])
            if precond == 1:
                rhs = rhs / D
            elif precond == 2:
                rhs = rhs * (xp / D)
            elif precond == 3:
                rhs = rhs * (np.maximum(xp, np.maximum(1e-5, ref)) / D)
            if dP is not None:
                rhs = rhs * dP
            if img_filter is not None and (kk < img_filter["K"] if img_filter["K"] > 0 else kk == 0):
                rhs = image_filter_fft(rhs, shape, img_filter["nf"], img_filter["F"])
            if kind == "PKMA" and (auto_relax or relax_scaling):
                xn, gn = np.linalg.norm(x), np.linalg.norm(rhs)
                if auto_relax:
                    if it == 0 and s == 0:
                        lam[0] = np.float32(xn / gn) * np.float32(0.25)
                    elif it > 0 and s == 0:
                        lam[it] = np.float32(lam[it - 1]) * np.float32(1.0 / (it / 35.0 + 1.0))
                if relax_scaling:
                    q = np.float32(xn / (gn * lam[it]))
                    if 0 < q < 1.5:
                        lam[it] = np.float32(lam[it]) * np.float32(q / 1.5)
                lm = float(lam[it])
            if kind == "PKMA":
                x = poisson_update("PKMA", x, rhs, lm, eps, float(alpha[it * S + s]), positivity)
            elif kind in ("MRAMLA", "MBSREM"):
                x = poisson_update("MBSREM", x, rhs, lm, eps, upper, positivity)
            elif ramla:
                x = poisson_update("BSREM", x, rhs, lm, eps, 0.0, positivity)
            else:
                x = x + lm * x / sens[s] * (rhs - sens[s])
        if mapstep:
            x = x - lm * x * prior_grad(x)
            x[x < eps] = eps
    return x


def loglik(y, fp, eps):
    """Poisson log-likelihood sum[y log(fp + eps) - (fp + eps)] in FP64."""
    f = np.asarray(fp, dtype=np.float64) + eps
    yy = np.asarray(y, dtype=np.float64)
    return float(np.sum(np.where(yy != 0, yy * np.log(f), 0.0) - f))


def ref_forward(geom: Geometry, image, subset, precision="double", threads=0):
    """The reference's own CPU projector (whole-sinogram subsets, PET)."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libref_siddon.so is not built")
    return _ref_call(L, geom, image, subset, True, precision, threads)


def ref_backward(geom: Geometry, y, subset, precision="double", threads=0, sens=False):
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libref_siddon.so is not built")
    return _ref_call(L, geom, y, subset, False, precision, threads, sens)


def _ref_call(L, geom, inp, subset, fp, precision, threads, sens=False):
    T = np.float64 if precision == "double" else np.float32
    fn = L.ref_siddon_d if precision == "double" else L.ref_siddon_f
    CT = ctypes.c_double if precision == "double" else ctypes.c_float
    P = ctypes.POINTER(CT)
    p = (lambda a: a.ctypes.data_as(P) if a is not None else None)
    n0, n1 = (0, geom.n_proj) if subset < 0 else (int(geom.n_meas[subset]), int(geom.n_meas[subset + 1]))
    xy = geom.xy.astype(T)
    z = np.ascontiguousarray(geom.z.astype(T)[n0 * 2:n1 * 2])
    inp = np.ascontiguousarray(inp, dtype=T).ravel()
    nmeas = geom.n_rows * geom.n_cols * (n1 - n0)
    out = np.zeros(nmeas * geom.nbins if fp else geom.n_img, dtype=T)
    s = np.zeros(geom.n_img, dtype=T) if sens else None
    tofc = geom.tofc.astype(T)
    fn(1 if fp else 0, geom.nx, geom.ny, geom.nz, *geom.d, *geom.b, geom.n_rows, geom.n_cols, n1 - n0, p(xy), p(z),
       p(inp), p(out), p(s), geom.nbins, geom.sigma_x, p(tofc), geom.global_factor, geom.epps, int(threads))
    return (out, s) if sens else out


def ref_corrected(geom: Geometry, inp, subset, fp, norm=None, atten=None, ct_atten=True, scat=None, threads=0,
                  sens=False):
    """The reference CPU projector (FP64) with PET corrections: norm / scat
    per measurement of the subset, atten an image (ct_atten) or per
    measurement.  Whole-sinogram subsets only."""
    L = ref_lib()
    P = ctypes.POINTER(ctypes.c_double)
    p = (lambda a: a.ctypes.data_as(P) if a is not None else None)
    n0, n1 = (0, geom.n_proj) if subset < 0 else (int(geom.n_meas[subset]), int(geom.n_meas[subset + 1]))
    xy = geom.xy.astype(np.float64)
    z = np.ascontiguousarray(geom.z.astype(np.float64)[n0 * 2:n1 * 2])
    inp = np.ascontiguousarray(inp, dtype=np.float64).ravel()
    nmeas = geom.n_rows * geom.n_cols * (n1 - n0)
    out = np.zeros(nmeas * geom.nbins if fp else geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    d = (lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel())
    norm, atten, scat = d(norm), d(atten), d(scat)
    tofc = geom.tofc.astype(np.float64)
    L.ref_siddon_corr_d(1 if fp else 0, geom.nx, geom.ny, geom.nz, *geom.d, *geom.b, geom.n_rows, geom.n_cols,
                        n1 - n0, p(xy), p(z), p(inp), p(out), p(s), geom.nbins, geom.sigma_x, p(tofc),
                        geom.global_factor, geom.epps, int(threads), p(norm), p(atten), 1 if ct_atten else 0, p(scat))
    return (out, s) if sens else out


def ref_multiray(geom: Geometry, inp, subset, fp, threads=0, sens=False):
    """The reference CPU projector (FP64) with geom.nr_xy x geom.nr_z rays per
    LOR over the crystal pitches geom.pitch.  Whole-sinogram subsets."""
    L = ref_lib()
    P = ctypes.POINTER(ctypes.c_double)
    p = (lambda a: a.ctypes.data_as(P) if a is not None else None)
    n0, n1 = (0, geom.n_proj) if subset < 0 else (int(geom.n_meas[subset]), int(geom.n_meas[subset + 1]))
    xy = geom.xy.astype(np.float64)
    z = np.ascontiguousarray(geom.z.astype(np.float64)[n0 * 2:n1 * 2])
    inp = np.ascontiguousarray(inp, dtype=np.float64).ravel()
    nmeas = geom.n_rows * geom.n_cols * (n1 - n0)
    out = np.zeros(nmeas * geom.nbins if fp else geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    tofc = geom.tofc.astype(np.float64)
    L.ref_multiray_d(1 if fp else 0, geom.nx, geom.ny, geom.nz, *geom.d, *geom.b, geom.n_rows, geom.n_cols, n1 - n0,
                     p(xy), p(z), p(inp), p(out), p(s), geom.nbins, geom.sigma_x, p(tofc), geom.global_factor,
                     geom.epps, int(threads), geom.nr_xy, geom.nr_z, geom.pitch[0], geom.pitch[1])
    return (out, s) if sens else out


def ref_listmode(geom: Geometry, inp, subset, fp, threads=0, sens=False):
    """The reference CPU projector (FP64) on the list-mode events of a subset."""
    L = ref_lib()
    P = ctypes.POINTER(ctypes.c_double)
    p = (lambda a: a.ctypes.data_as(P) if a is not None else None)
    e0, e1 = (0, geom.n_proj) if subset < 0 else (int(geom.n_meas[subset]), int(geom.n_meas[subset + 1]))
    xyz = np.ascontiguousarray(geom.xy.astype(np.float64)[e0 * 6:e1 * 6])
    inp = np.ascontiguousarray(inp, dtype=np.float64).ravel()
    out = np.zeros(e1 - e0 if fp else geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    L.ref_listmode_d(1 if fp else 0, geom.nx, geom.ny, geom.nz, *geom.d, *geom.b, e1 - e0, p(xyz), p(inp), p(out), p(s),
                     geom.global_factor, geom.epps, int(threads))
    return (out, s) if sens else out


def ref_orth(geom: Geometry, inp, subset, fp, proj_type, sens=False, norm=None, atten=None, threads=0):
    """The reference CPU projector (FP64) with projector type 2 or 3 on
    whole-sinogram subsets.  The voxel-centre arrays it indexes are padded
    with far-away sentinels on both sides: it reads one centre past the end
    of a slice and rows outside the grid at the ends of the tube."""
    L = ref_lib()
    P = ctypes.POINTER(ctypes.c_double)
    p = (lambda a: a.ctypes.data_as(P) if a is not None else None)
    n0, n1 = (0, geom.n_proj) if subset < 0 else (int(geom.n_meas[subset]), int(geom.n_meas[subset + 1]))
    xy = geom.xy.astype(np.float64)
    z = np.ascontiguousarray(geom.z.astype(np.float64)[n0 * 2:n1 * 2])
    inp = np.ascontiguousarray(inp, dtype=np.float64).ravel()
    nmeas = geom.n_rows * geom.n_cols * (n1 - n0)
    out = np.zeros(nmeas * geom.nbins if fp else geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    pad = 64
    centres = []
    for n, b, d in zip((geom.nx, geom.ny, geom.nz), geom.b, geom.d):
        c = np.full(n + 2 * pad, 1e12, dtype=np.float64)
        c[pad:pad + n] = b + d * np.arange(n, dtype=np.float64) + d / 2.0
        centres.append(c)
    cp = [c.ctypes.data_as(P) for c in centres]
    cp = [ctypes.cast(ctypes.addressof(q.contents) + pad * 8, P) for q in cp]
    # the reference indexes the table up to (bmax - bmin) * 1000, past its last entry when entries
    # were dropped; the padding repeats the last entry there, as the restatement reads it
    V = np.concatenate([geom.V.astype(np.float64), np.full(4096, geom.V[-1], dtype=np.float64)])
    d64 = (lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel())
    norm, atten = d64(norm), d64(atten)
    tofc = geom.tofc.astype(np.float64)
    width = geom.tube_width if proj_type == 2 else geom.tube_radius
    L.ref_orth_d(1 if fp else 0, geom.nx, geom.ny, geom.nz, *geom.d, *geom.b, geom.n_rows, geom.n_cols, n1 - n0,
                 p(xy), p(z), p(inp), p(out), p(s), geom.nbins, geom.sigma_x, p(tofc), geom.global_factor, geom.epps,
                 int(threads), proj_type, width, cp[0], cp[1], cp[2], geom.vol[0], geom.vol[1], geom.vol[2], p(V),
                 p(norm), p(atten))
    del centres
    return (out, s) if sens else out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


# ---------------------------------------------------------------------------
# Projector type 5 (branchless distance-driven), CT
# ---------------------------------------------------------------------------

def _ct_struct(geom: Geometry, subset):
    g = OracleCT()
    g.nx, g.ny, g.nz = geom.nx, geom.ny, geom.nz
    g.dx, g.dy, g.dz = geom.d
    g.bx, g.by, g.bz = geom.b
    g.n_rows, g.n_cols = geom.n_rows, geom.n_cols
    g.proj0 = 0 if subset < 0 else int(geom.n_meas[subset])
    g.n_proj = geom.n_proj if subset < 0 else int(geom.n_meas[subset + 1] - geom.n_meas[subset])
    g.pitch_x, g.pitch_y = geom.pitch
    g.xy = geom.xy.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    g.uv = geom.z.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    return g


def bdd_forward(geom: Geometry, image, subset):
    """FP64 branchless distance-driven forward projection of one subset."""
    img = np.ascontiguousarray(image, dtype=np.float64).ravel()
    g = _ct_struct(geom, subset)
    y = np.zeros(geom.rays(subset), dtype=np.float64)
    if lib().oracle_bdd_fp(ctypes.byref(g), _dp(img), _dp(y)) != 0:
        raise MemoryError("oracle_bdd_fp")
    return y


def bdd_backward(geom: Geometry, y, subset, sens=False):
    """FP64 voxel-driven distance-driven backprojection (and its weight sum)."""
    yy = np.ascontiguousarray(y, dtype=np.float64).ravel()
    g = _ct_struct(geom, subset)
    img = np.zeros(geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    if lib().oracle_bdd_bp(ctypes.byref(g), _dp(yy), _dp(img), _dp(s)) != 0:
        raise MemoryError("oracle_bdd_bp")
    return (img, s) if sens else img


def bdd_backward_ray(geom: Geometry, y, subset, sens=False):
    """FP64 ray-driven distance-driven backprojection: the exact adjoint of
    bdd_forward (and its A^T 1)."""
    yy = np.ascontiguousarray(y, dtype=np.float64).ravel()
    g = _ct_struct(geom, subset)
    img = np.zeros(geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    if lib().oracle_bdd_bp_ray(ctypes.byref(g), _dp(yy), _dp(img), _dp(s)) != 0:
        raise MemoryError("oracle_bdd_bp_ray")
    return (img, s) if sens else img


def tv_gradient(u, shape, smooth, beta):
    """Smoothed TV gradient of auxKernels.cl:1733-1990 (TVKernel, plain TV,
    no reference image) with the edge-clamped neighbours of its texture path,
    in FP64.  ``u`` is Fortran-ordered, ``shape`` = (Nx, Ny, Nz)."""
    nx, ny, nz = shape
    U = np.asarray(u, dtype=np.float64).reshape((nx, ny, nz), order="F")

    def sh(a, dx=0, dy=0, dz=0):
        ix = np.clip(np.arange(nx) + dx, 0, nx - 1)
        iy = np.clip(np.arange(ny) + dy, 0, ny - 1)
        iz = np.clip(np.arange(nz) + dz, 0, nz - 1)
        return a[ix][:, iy][:, :, iz]

    uPx, uPy, uPz = sh(U, 1), sh(U, 0, 1), sh(U, 0, 0, 1)
    uMx, uMy, uMz = sh(U, -1), sh(U, 0, -1), sh(U, 0, 0, -1)
    uix, uiy = sh(U, -1, 1), sh(U, -1, 0, 1)
    ujx, ujy = sh(U, 1, -1), sh(U, 0, -1, 1)
    ukx, uky = sh(U, 1, 0, -1), sh(U, 0, 1, -1)

    def sq(a, b, c):
        return np.sqrt(a * a + b * b + c * c + smooth)

    p0 = sq(uPx - U, uPy - U, uPz - U)
    p1 = sq(U - uMx, uix - uMx, uiy - uMx)
    p2 = sq(ujx - uMy, U - uMy, ujy - uMy)
    p3 = sq(ukx - uMz, uky - uMz, U - uMz)
    g = (3 * U - uPx - uPy - uPz) / p0 + (U - uMx) / p1 + (U - uMy) / p2 + (U - uMz) / p3 + 1e-7
    return (beta * g).ravel(order="F")


def power_method(geom: Geometry, n_iter, seed=0, x0=None):
    """Largest eigenvalue of A^T A by power iteration (functions.hpp:2417-2540)."""
    if x0 is None:
        rng = np.random.default_rng(seed)
        x = np.abs(rng.standard_normal(geom.n_img))
    else:
        x = np.asarray(x0, dtype=np.float64).copy()
    x /= np.linalg.norm(x)
    L = 0.0
    for _ in range(n_iter):
        r = bdd_backward(geom, bdd_forward(geom, x, -1), -1)
        L = float(np.dot(x, r) / np.dot(x, x))
        x = r / np.linalg.norm(r)
    return L


def row_filter_fft(v, rows, nf, filt, inverse=False):
    """filtering / filteringInverse (functions.hpp:1882-1952) in FP64: each
    column of `rows` values zero-padded to nf, its FFT multiplied (divided)
    by the real filter, transformed back, the real part cut to `rows`."""
    V = np.asarray(v, dtype=np.float64).reshape(-1, rows).T
    F = np.fft.fft(V, n=nf, axis=0)
    f = np.asarray(filt, dtype=np.float64)[:, None]
    F = F / f if inverse else F * f
    return np.real(np.fft.ifft(F, axis=0))[:rows].T.ravel()


def image_filter_fft(g, shape, nf, F):
    """filtering2D (functions.hpp:1908-1932) in FP64: every slice of g
    zero-padded to nf x nf, its 2-D FFT multiplied by the real filter F,
    transformed back, the real part cut to nx x ny."""
    nx, ny, _ = shape
    G = np.asarray(g, dtype=np.float64).reshape(shape, order='F')
    T = np.fft.fft2(G, s=(nf, nf), axes=(0, 1)) * np.asarray(F, dtype=np.float64)[:, :, None]
    return np.real(np.fft.ifft2(T, axes=(0, 1)))[:nx, :ny, :].ravel(order='F')


def pdhg_tv(geom: Geometry, y, x0, n_iter, tau, beta, smooth, sigma=1.0, theta=1.0, eps=1e-5,
            positivity=True, tv_grad=None, prox=None, meas_filter=None, tgv=None, img_filter=None):
    """PDHG with a TV-gradient term, one subset (computeForwardProject.h:227-316,
    algorithms.h:329-420, auxKernels.cl:2034-2062), in FP64.  tv_grad(x), when
    given, replaces the plain TV term beta * dTV(x) (the other TVKernel forms).
    prox = dict(sigma2=..., l2=..., diff_type=...): the proximal TV instead
    (priors.h:261-281), a dual variable q on the beta ball, rhs -= div q.
    meas_filter = dict(filter0, ffilter, nf, rows, K, tau2): the filtering-based
    measurement preconditioner (computeForwardProject.h:21-45, 253-298): the
    residual filtered by filter0; for k < K the dual step (p + sigma F r)
    divided by ffilter in the Fourier domain, from k = K on the plain dual
    step without filtering and the primal step tau2 (K = 0: every residual
    filtered, plain dual step).  tgv = dict(alpha0, alpha1, sigma2, l2,
    three_d): TGV instead of the TV term (priors.h:284-313,
    image_oracle.proxtgv_step with theta and the current tau), the plain
    dual step divided by 1 + sigma beta (computeForwardProject.h:295-298;
    with meas_filter, its ffilter built from sigma beta).  img_filter =
    dict(nf, F, K, tau2): the filtering-based image preconditioner, A^T p plus
    the TV term filtered (image_filter_fft) in iterations k < K (K = 0: k = 0
    only) and the primal step tau2 from k = K on (subiterStep.h:28-45)."""
    from oracle import image_oracle as io
    shape = (geom.nx, geom.ny, geom.nz)
    x = np.asarray(x0, dtype=np.float64).copy()
    u = x.copy()
    p = np.zeros(geom.rays(-1), dtype=np.float64)
    q = np.zeros((3, geom.n_img))
    if tgv is not None:
        three_d = tgv.get("three_d", True)
        r_t = np.zeros((6 if three_d else 3, geom.n_img))
        v_t = np.zeros((3 if three_d else 2, geom.n_img))
    den = 1.0 + sigma * (beta if tgv is not None else 1.0)
    yy = np.asarray(y, dtype=np.float64)
    for k in range(n_iter):
        res = bdd_forward(geom, x, -1) - yy
        mf = meas_filter
        if mf is not None and mf["K"] > 0 and k == mf["K"]:
            tau = mf["tau2"]
        if img_filter is not None and img_filter["K"] > 0 and k == img_filter["K"]:
            tau = img_filter["tau2"]
        if mf is not None and (mf["K"] == 0 or k < mf["K"]):
            r = row_filter_fft(res, mf["rows"], mf["nf"], mf["filter0"])
            if mf["K"] == 0:
                p = (p + sigma * r) / den
            else:
                p = row_filter_fft(p + sigma * r, mf["rows"], mf["nf"], mf["ffilter"], inverse=True)
        else:
            p = (p + sigma * res) / den
        if tgv is not None:
            q, r_t, v_t, rhs = io.proxtgv_step(x, q, r_t, v_t, bdd_backward(geom, p, -1), shape, tgv["sigma2"],
                                               tgv["alpha0"], tgv["alpha1"], theta, tau, tgv.get("l2", True),
                                               three_d)
        elif prox is not None:
            q = io.proxtv_dual(x, q, shape, prox["sigma2"], beta, prox.get("l2", True), prox.get("diff_type", 0))
            rhs = bdd_backward(geom, p, -1) - io.proxtv_divergence(q, shape, prox.get("diff_type", 0))
        else:
            rhs = bdd_backward(geom, p, -1) + (tv_gradient(x, shape, smooth, beta) if tv_grad is None else tv_grad(x))
        if img_filter is not None and (k < img_filter["K"] if img_filter["K"] > 0 else k == 0):
            rhs = image_filter_fft(rhs, shape, img_filter["nf"], img_filter["F"])
        u_prev = u.copy()
        u = u - tau * rhs
        if positivity:
            u = np.maximum(eps, u)
        x = u + theta * (u - u_prev)
    return x


# ---------------------------------------------------------------------------
# Projector type 4 (interpolation), PET and CT
# ---------------------------------------------------------------------------

def interp_forward(geom: Geometry, image, subset):
    """FP64 type-4 forward projection (ray-marched trilinear samples) of one
    subset; all TOF bins, bin-major."""
    img = np.ascontiguousarray(image, dtype=np.float64).ravel()
    g = geom.struct(subset)
    y = np.zeros(geom.rays(subset) * geom.nbins, dtype=np.float64)
    if lib().oracle_interp_fp(ctypes.byref(g), geom.dL, _dp(img), _dp(y)) != 0:
        raise ValueError("oracle_interp_fp")
    return y


def interp_backward(geom: Geometry, y, subset, sens=False):
    """FP64 type-4 PET backprojection (nearest voxel per sample); y=None
    backprojects ones."""
    g = geom.struct(subset)
    img = np.zeros(geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    yy = None if y is None else np.ascontiguousarray(y, dtype=np.float64).ravel()
    if lib().oracle_interp_bp(ctypes.byref(g), geom.dL, _dp(yy), _dp(img), _dp(s)) != 0:
        raise ValueError("oracle_interp_bp")
    return (img, s) if sens else img


def interp_ct_backward(geom: Geometry, y, subset, sens=False):
    """FP64 type-4 CT backprojection (voxel driven, bilinear detector samples)."""
    yy = np.ascontiguousarray(y, dtype=np.float64).ravel()
    g = _ct_struct(geom, subset)
    img = np.zeros(geom.n_img, dtype=np.float64)
    s = np.zeros(geom.n_img, dtype=np.float64) if sens else None
    if lib().oracle_interp_ct_bp(ctypes.byref(g), geom.kerroin, _dp(yy), _dp(img), _dp(s)) != 0:
        raise ValueError("oracle_interp_ct_bp")
    return (img, s) if sens else img
