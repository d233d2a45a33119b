"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run where the OMEGA sources are, with $OMEGA_REFERENCE naming their root:

    OMEGA_REFERENCE=<checkout> python tests/golden/make_golden.py   # everything
    python tests/golden/make_golden.py volumes    # the type-3 tables only
    python tests/golden/make_golden.py nlm        # the NLM patch weights only
    python tests/golden/make_golden.py tv         # the anatomical TV preparation only
    python tests/golden/make_golden.py ramp       # the measurement filters only
    python tests/golden/make_golden.py geom NAME  # one geometry fixture

For every option set in configs.py it imports the reference's own Python
projector surface (omegatomo.projector.proj.projectorClass), runs its
addProjector(), and stores the geometry arrays it produces (detector
coordinates, subset indices, measurement counts, voxel grid) in
``geom_<name>.npz``.  For the small PET sets it also runs the reference's own
OpenMP CPU projector (projectorType123Implementation4<double>, compiled by
oracle/Makefile into oracle/_ref/libref_siddon.so) on a seeded image and a
seeded measurement vector and stores the results in ``proj_<name>.npz``.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("OMEGA_REFERENCE", "")
sys.path.insert(0, HERE)
from configs import CONFIGS, GEOMETRY_KEYS, SCALAR_KEYS, SCALE_KEYS, _pet, apply  # noqa: E402

PROJ_SETS = ["pet_mini", "pet_tof_small"]
# small TOF set for projector fixtures (kept separate to keep the files small)
CONFIGS_EXTRA = {
    "pet_tof_small": _pet(8, 8, 6, 300, 24, 32, 24, 11, 180, 26, subsets=4, TOF_bins=7, TOF_bins_used=7,
                          TOF_FWHM=200e-12, TOF_width=CONFIGS["pet_mini_tof"]["TOF_width"]),
}


def reference_projector():
    if not REF:
        sys.exit("set OMEGA_REFERENCE to the root of an OMEGA checkout (the directory holding source/Python)")
    sys.path.insert(0, os.path.join(REF, "source", "Python"))
    from omegatomo.projector import proj
    return proj


def geometry(proj, cfg):
    o = apply(proj.projectorClass(), cfg)
    o.addProjector()
    out = {}
    for k in GEOMETRY_KEYS:
        out[k] = np.asarray(getattr(o, k))
    for k in SCALAR_KEYS:
        out["s_" + k] = np.asarray(getattr(o, k))
    if o.projector_type in (4, 5, 14, 41, 15, 45, 54, 51):
        for k in SCALE_KEYS:
            out["p_" + k] = np.asarray(getattr(o, k))
    if o.TOF:
        out["TOFCenter"] = np.asarray(o.TOFCenter)
    if o.CT:
        out["uV"] = np.asarray(o.uV)
    return o, out


def ref_cpu_lib():
    path = os.path.join(REPO, "oracle", "_ref", "libref_siddon.so")
    if not os.path.exists(path):
        raise SystemExit("build the reference CPU projector first: make -C oracle")
    L = ctypes.CDLL(path)
    D = ctypes.c_double
    P = ctypes.POINTER(ctypes.c_double)
    u = ctypes.c_uint32
    L.ref_siddon_d.argtypes = [ctypes.c_int, u, u, u, D, D, D, D, D, D, u, u, u, P, P, P, P, P, u, D, P, D, D, u]
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def ref_project(L, o, subset, fp, inp, sens=False):
    """Runs the reference CPU projector on one whole-sinogram subset."""
    nb = int(o.TOF_bins_used) if o.TOF else 1
    n0, n1 = int(o.nMeas[subset]), int(o.nMeas[subset + 1])
    nproj = n1 - n0
    xy = np.ascontiguousarray(o.x.astype(np.float64).ravel())
    z = np.ascontiguousarray(o.z.astype(np.float64).ravel()[n0 * 2:n1 * 2])
    N = int(o.Nx[0]) * int(o.Ny[0]) * int(o.Nz[0])
    nmeas = int(o.nRowsD) * int(o.nColsD) * nproj
    inp = np.ascontiguousarray(inp, dtype=np.float64)
    out = np.zeros(nmeas * nb if fp else N, dtype=np.float64)
    s = np.zeros(N, dtype=np.float64) if sens else None
    tofc = np.ascontiguousarray(np.asarray(o.TOFCenter, dtype=np.float64)) if o.TOF else None
    L.ref_siddon_d(1 if fp else 0, int(o.Nx[0]), int(o.Ny[0]), int(o.Nz[0]), float(o.dx[0]), float(o.dy[0]),
                   float(o.dz[0]), float(o.bx[0]), float(o.by[0]), float(o.bz[0]), int(o.nRowsD), int(o.nColsD),
                   nproj, _p(xy), _p(z), _p(inp), _p(out), _p(s), nb, float(o.sigma_x), _p(tofc),
                   float(o.global_factor), float(o.epps), 0)
    return out, s


def psf_fixture(proj):
    """The reference's PSF window (proj.py PSFKernel, run by its addProjector)
    for pet_mini with FWHM 4 x 4 x 6 mm, stored in psf_pet_mini.npz."""
    o = apply(proj.projectorClass(), dict(CONFIGS["pet_mini"], use_psf=True, FWHM=np.array([4., 4., 6.])))
    o.addProjector()
    out = {"gaussK": np.asarray(o.gaussK, dtype=np.float32).ravel(order='F'),
           "g_dim": np.array([o.g_dim_x, o.g_dim_y, o.g_dim_z], dtype=np.int64), "FWHM": np.array([4., 4., 6.])}
    np.savez_compressed(os.path.join(HERE, "psf_pet_mini.npz"), **out)
    print("psf_pet_mini", out["g_dim"], out["gaussK"].shape)


def prior_weight_fixture(proj):
    """The reference's neighbourhood weights (prepass.py computeWeights +
    quadWeights / huberWeights) for pet_mini with Ndx = Ndy = Ndz = 1 and
    Ndx = Ndy = 2, Ndz = 1, stored in priorw_pet_mini.npz."""
    # prepass.py loaded on its own: the package's __init__ imports a module
    # that does not parse under Python 3.12 (mixed tabs in recomain.py)
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "omega_prepass", os.path.join(REF, "source", "Python", "omegatomo", "reconstruction", "prepass.py"))
    prepass = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(prepass)
    out = {}
    for tag, nd in (("111", (1, 1, 1)), ("221", (2, 2, 1))):
        o = apply(proj.projectorClass(), CONFIGS["pet_mini"])
        o.addProjector()
        o.Ndx, o.Ndy, o.Ndz = nd
        o.weights = np.empty(0, dtype=np.float32)
        o.GGMRF = False
        prepass.computeWeights(o, False)
        w = np.asarray(o.weights, dtype=np.float32).copy()
        prepass.quadWeights(o, True)
        out["quad_" + tag] = np.asarray(o.weights_quad, dtype=np.float32)
        o.weights = w
        o.weights_huber = np.empty(0, dtype=np.float32)
        prepass.huberWeights(o)
        out["huber_" + tag] = np.asarray(o.weights_huber, dtype=np.float32)
        out["weights_" + tag] = w
    # GGMRF: the branch of computeWeights for it and quadWeights with options.GGMRF set
    o = apply(proj.projectorClass(), CONFIGS["pet_mini"])
    o.addProjector()
    o.Ndx = o.Ndy = o.Ndz = 1
    o.weights = np.empty(0, dtype=np.float32)
    o.GGMRF = True
    prepass.computeWeights(o, True)
    prepass.quadWeights(o, True)
    out["ggmrf_111"] = np.asarray(o.weights_quad, dtype=np.float32)
    # weighted mean: weightedWeights on the distance weights
    o = apply(proj.projectorClass(), CONFIGS["pet_mini"])
    o.addProjector()
    o.Ndx = o.Ndy = o.Ndz = 1
    o.weights = np.empty(0, dtype=np.float32)
    o.GGMRF = False
    prepass.computeWeights(o, False)
    o.weighted_weights = np.empty(0, dtype=np.float32)
    prepass.weightedWeights(o)
    out["wmean_111"] = np.asarray(o.weighted_weights, dtype=np.float32).ravel(order='F')
    np.savez_compressed(os.path.join(HERE, "priorw_pet_mini.npz"), **out)
    print("priorw_pet_mini", {k: v.shape for k, v in out.items()})


def volume_fixture():
    """The reference's type-3 table (coordinates.py computeVoxelVolumes) for
    two tube / voxel sizes, stored in vol_tables.npz."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "omega_coordinates", os.path.join(REF, "source", "Python", "omegatomo", "projector", "coordinates.py"))
    coords = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(coords)

    class Opt:
        pass
    out = {}
    for tag, (R, r, d) in VOLUME_CASES.items():
        o = Opt()
        o.projector_type = 3
        o.tube_radius, o.voxel_radius = R, r
        o.dx, o.dy, o.dz = (np.array([v], dtype=np.float32) for v in d)
        coords.computeVoxelVolumes(o)
        out["V_" + tag] = np.asarray(o.V, dtype=np.float32)
        out["s_" + tag] = np.array([o.bmin, o.bmax, o.Vmax, o.voxel_radius], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "vol_tables.npz"), **out)
    print("vol_tables", {k: v.shape for k, v in out.items()})


def nlm_fixture():
    """The reference's NLM patch weights (prepass.py NLMPrepass) for two patch
    sizes, stored in nlm_gauss.npz."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "omega_prepass", os.path.join(REF, "source", "Python", "omegatomo", "reconstruction", "prepass.py"))
    prepass = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(prepass)

    class Opt:
        pass
    out = {}
    for tag, (nl, sd) in {"111": ((1, 1, 1), 2.0), "221": ((2, 2, 1), 1.5)}.items():
        o = Opt()
        o.Nlx, o.Nly, o.Nlz = nl
        o.NLM_gauss = sd
        o.NLM_use_anatomical = False
        prepass.NLMPrepass(o)
        out["g_" + tag] = np.asarray(o.gaussianNLM, dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "nlm_gauss.npz"), **out)
    print("nlm_gauss", {k: v.shape for k, v in out.items()})


def tv_fixture():
    """The reference's anatomical TV preparation (prepass.py TVPrepass): the
    min-max normalised reference image (TVtype 2) and the 9-channel weighting
    tensor of TVtype 1 (assembleS), for a seeded 7 x 6 x 5 reference image
    with a constant block (zero gradients), stored in tv_anat.npz.  Its
    image resize is never reached (the image has the reconstruction's size),
    so a stand-in skimage module satisfies the import."""
    import importlib.util
    import types
    for name in ("skimage", "skimage.transform"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["skimage.transform"].resize = None
    spec = importlib.util.spec_from_file_location(
        "omega_prepass", os.path.join(REF, "source", "Python", "omegatomo", "reconstruction", "prepass.py"))
    prepass = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(prepass)

    class Opt:
        pass
    rng = np.random.default_rng(77)
    shape = (7, 6, 5)
    img = rng.uniform(2.0, 9.0, shape).astype(np.float32)
    img[1:4, 1:4, 1:3] = 5.0
    img = np.asfortranarray(img)
    out = {"ref": img}
    for tvtype, T in ((1, 0.3), (2, 0.3), (1, 2.0)):
        o = Opt()
        o.Nx, o.Ny, o.Nz = (np.array([v], dtype=np.uint32) for v in shape)
        o.TV_use_anatomical = True
        o.TVtype = tvtype
        o.T = T
        o.TV_referenceImage = img.copy(order="F")
        prepass.TVPrepass(o)
        if tvtype == 1:
            out[f"s_T{T}"] = np.asarray(o.s, dtype=np.float32)
        out["ref_norm"] = np.asarray(o.TV_referenceImage, dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "tv_anat.npz"), **out)
    print("tv_anat", {k: v.shape for k, v in out.items()})


def ramp_fixture():
    """The reference's rampFilt (omegatomo/reconstruction/rampfilt.py) for
    every window, two cut-offs and even / odd lengths, stored in
    ramp_filters.npz (key window_c_N)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "omega_rampfilt", os.path.join(REF, "source", "Python", "omegatomo", "reconstruction", "rampfilt.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for window in ("hamming", "hann", "blackman", "nuttal", "gaussian", "shepp-logan", "cosine", "parzen", "none"):
        for c in (1.0, 0.8):
            for N in (512, 64, 101):
                out[f"{window}_{c}_{N}"] = np.asarray(mod.rampFilt(N, window, c, 0.25))
    # the 2-D form (use2D) of the image preconditioner: its shape and the
    # first N^2 values, which the library reads as the N x N filter
    for N in (16, 32):
        f2 = np.asarray(mod.rampFilt(N, "hamming", 1.0, 0.25, True))
        out[f"use2D_shape_{N}"] = np.asarray(f2.shape)
        out[f"use2D_first_{N}"] = np.ascontiguousarray(f2).ravel()[:N * N].copy()
    np.savez_compressed(os.path.join(HERE, "ramp_filters.npz"), **out)
    print("ramp_filters", len(out))


# type-3 table cases: tube radius, voxel radius (before scaling), voxel size (dx, dy, dz)
VOLUME_CASES = {"a": (1.0, 1.0, (2.0, 2.0, 2.5)), "b": (2.5, 1.0, (1.5, 1.5, 1.5))}


def main():
    if sys.argv[1:] == ["volumes"]:
        volume_fixture()
        return
    if sys.argv[1:] == ["nlm"]:
        nlm_fixture()
        return
    if sys.argv[1:] == ["ramp"]:
        ramp_fixture()
        return
    if sys.argv[1:] == ["tv"]:
        tv_fixture()
        return
    if sys.argv[1:] == ["priorw"]:
        prior_weight_fixture(reference_projector())
        return
    if sys.argv[1:2] == ["geom"]:
        proj = reference_projector()
        for name in sys.argv[2:]:
            _, g = geometry(proj, CONFIGS[name])
            np.savez_compressed(os.path.join(HERE, f"geom_{name}.npz"), **g)
        return
    proj = reference_projector()
    volume_fixture()
    nlm_fixture()
    tv_fixture()
    ramp_fixture()
    psf_fixture(proj)
    prior_weight_fixture(proj)
    allc = dict(CONFIGS)
    allc.update(CONFIGS_EXTRA)
    L = None
    for name, cfg in allc.items():
        o, g = geometry(proj, cfg)
        np.savez_compressed(os.path.join(HERE, f"geom_{name}.npz"), **g)
        print(name, {k: np.shape(v) for k, v in g.items() if np.ndim(v) > 0})
        if name in PROJ_SETS:
            L = L or ref_cpu_lib()
            rng = np.random.default_rng(1234)
            N = int(o.N[0])
            img = rng.uniform(0.5, 1.5, N)
            fixtures = {"image": img.astype(np.float32)}
            nb = int(o.TOF_bins_used) if o.TOF else 1
            subsets = [0, int(o.subsets) - 1] if nb == 1 else [0]
            for s in subsets:
                y, _ = ref_project(L, o, s, True, img.astype(np.float32).astype(np.float64))
                fixtures[f"fp_{s}"] = y.astype(np.float32)
            m = int(o.nMeasSubset[0, 0]) * nb
            yin = rng.uniform(0.0, 2.0, m)
            fixtures["bp_in_0"] = yin.astype(np.float32)
            bp, sens = ref_project(L, o, 0, False, yin.astype(np.float32).astype(np.float64), sens=True)
            fixtures["bp_0"] = bp.astype(np.float32)
            fixtures["sens_0"] = sens.astype(np.float32)
            np.savez_compressed(os.path.join(HERE, f"proj_{name}.npz"), **fixtures)
            print("  projector fixtures:", list(fixtures))


if __name__ == "__main__":
    main()
