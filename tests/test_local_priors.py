"""Local priors: the median root prior (its median pinned against the
reference's CPU medianFilter3D, oracle/_ref MRP.h), the TV prior of the MAP
algorithms and GGMRF (weights pinned against the reference's prepass,
golden priorw_pet_mini.npz): CUDA gradients against the restatements and
OSL-OSEM / BSREM with each prior."""
import ctypes

import numpy as np
import pytest

from oracle import image_oracle as io
from oracle import oracle as orc

SHAPE = (12, 11, 9)


@pytest.mark.parametrize("m", [(1, 1, 1), (2, 1, 1), (1, 1, 0)])
def test_median_matches_reference(m):
    if orc.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    L = orc.ref_lib()
    P = ctypes.POINTER(ctypes.c_double)
    i32 = ctypes.c_int32
    L.ref_median_d.argtypes = [P, P, i32, i32, i32, i32, i32, i32]
    rng = np.random.default_rng(sum(m))
    u = np.round(rng.uniform(0.5, 1.5, int(np.prod(SHAPE))), 2)   # rounded: ties in most windows
    pad = io.padded_symmetric(u, SHAPE, m)
    med = np.zeros(u.size)
    L.ref_median_d(pad.ctypes.data_as(P), med.ctypes.data_as(P), *SHAPE, *m)
    # the restatement's gradient with no_norm and beta 1 is u - median
    got = u - io.mrp_gradient(u, SHAPE, m, 1.0, 1e-8, no_norm=True)
    assert np.array_equal(got, med)


@pytest.mark.gpu
@pytest.mark.parametrize("m,no_norm", [((1, 1, 1), False), ((2, 1, 1), True), ((1, 1, 0), False)])
def test_kernel_matches_restatement(cuda, m, no_norm):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(3)
    n = int(np.prod(SHAPE))
    u = np.round(rng.uniform(0.5, 1.5, n), 2).astype(np.float32)
    U = torch.tensor(u, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_mrp_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE, *m,
                 1e-8, 0.3, 1 if no_norm else 0, _stream(cuda))
    want = 0.5 + io.mrp_gradient(u.astype(np.float64), SHAPE, m, 0.3, 1e-8, no_norm=no_norm)
    assert np.max(np.abs(out.cpu().numpy() - want)) < 1e-6


@pytest.mark.gpu
def test_builtin_osl_osem_with_mrp(cuda):
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(8)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.OSL_OSEM = True
    o.MRP = True
    o.beta = 0.01
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    nd = (int(o.Ndx), int(o.Ndy), int(o.Ndz))
    ref = orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=lambda v: io.mrp_gradient(v, shape, nd, 0.01, g.epps))
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.osem(g, ys, np.ones(g.n_img), 2)) > 1e-4


@pytest.mark.gpu
def test_tv_gradient_kernel_matches_oracle(cuda):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(4)
    n = int(np.prod(SHAPE))
    u = rng.uniform(0.5, 1.5, n).astype(np.float32)
    U = torch.tensor(u, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_tv_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE, 0.3,
                 1e-4, _stream(cuda))
    want = 0.5 + orc.tv_gradient(u.astype(np.float64), SHAPE, 1e-4, 0.3)
    assert orc.rel_l2(out.cpu().numpy() - 0.5, want - 0.5) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["OSL_OSEM", "BSREM"])
def test_builtin_with_tv_prior(cuda, method):
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(9)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    setattr(o, method, True)
    o.TV = True
    o.TVsmoothing = 1e-2
    o.beta = 0.002
    o.Niter = 2
    lam = np.array([0.2, 0.12], np.float32)
    if method == "BSREM":
        o.lambdaN = lam
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)

    def grad(v):
        return orc.tv_gradient(v, shape, 1e-2, 0.002)
    if method == "OSL_OSEM":
        ref = orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=grad)
    else:
        ref = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam, prior_grad=grad)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)


def test_ggmrf_weights_match_reference():
    from conftest import make_options
    from omega_b200 import priors
    import os
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "priorw_pet_mini.npz"))
    o = make_options("pet_mini")
    o.Ndx = o.Ndy = o.Ndz = 1
    assert np.array_equal(priors.ggmrf_weights(o), f["ggmrf_111"])


@pytest.mark.gpu
def test_ggmrf_kernel_matches_restatement(cuda):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(5)
    n = int(np.prod(SHAPE))
    u = np.round(rng.uniform(0.5, 1.5, n), 2).astype(np.float32)     # equal neighbours: the d = 0 skip
    w = rng.uniform(0.01, 0.1, 26).astype(np.float32)
    U, W = torch.tensor(u, device=cuda), torch.tensor(w, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_ggmrf_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE,
                 1, 1, 1, ctypes.c_void_p(W.data_ptr()), 2.0, 1.5, 0.05, 0.3, _stream(cuda))
    want = 0.5 + io.ggmrf_gradient(u.astype(np.float64), SHAPE, (1, 1, 1), w.astype(np.float64), 2.0, 1.5, 0.05, 0.3)
    assert orc.rel_l2(out.cpu().numpy() - 0.5, want - 0.5) < 2e-5


@pytest.mark.gpu
def test_builtin_osl_osem_with_ggmrf(cuda):
    from conftest import make_options
    from omega_b200 import priors
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(10)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.OSL_OSEM = True
    o.GGMRF = True
    o.GGMRF_p, o.GGMRF_q, o.GGMRF_c = 2.0, 1.5, 0.05
    o.beta = 0.005
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    w = priors.ggmrf_weights(o).astype(np.float64)
    ref = orc.osem(g, ys, np.ones(g.n_img), 2,
                   prior_grad=lambda v: io.ggmrf_gradient(v, shape, (1, 1, 1), w, 2.0, 1.5, 0.05, 0.005))
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.osem(g, ys, np.ones(g.n_img), 2)) > 1e-4


@pytest.mark.gpu
def test_builtin_bsrem_with_hyperbolic(cuda):
    import torch
    from conftest import make_options
    from omega_b200 import _native, priors
    from omega_b200 import reconstruction as rec
    from omega_b200.reconstruction import _stream
    # the kernel alone
    rng = np.random.default_rng(12)
    n = int(np.prod(SHAPE))
    u = rng.uniform(0.5, 1.5, n).astype(np.float32)
    w = rng.uniform(0.01, 0.1, 26).astype(np.float32)
    U, W = torch.tensor(u, device=cuda), torch.tensor(w, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_hyperbolic_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE,
                 1, 1, 1, ctypes.c_void_p(W.data_ptr()), 0.2, 0.3, _stream(cuda))
    want = 0.5 + io.hyperbolic_gradient(u.astype(np.float64), SHAPE, (1, 1, 1), w.astype(np.float64), 0.2, 0.3)
    assert orc.rel_l2(out.cpu().numpy() - 0.5, want - 0.5) < 1e-5
    # BSREM with it
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.BSREM = True
    o.hyperbolic = True
    o.hyperbolicDelta = 0.1
    o.beta = 0.05
    o.Niter = 2
    lam = np.array([0.2, 0.12], np.float32)
    o.lambdaN = lam
    res, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    wq = priors.normalised_weights(priors.neighbourhood_weights(o)).astype(np.float64)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam,
                      prior_grad=lambda v: io.hyperbolic_gradient(v, shape, (1, 1, 1), wq, 0.1, 0.05))
    x = res.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.relaxed(g, ys, np.ones(g.n_img), 2, "RAMLA", lam=lam)) > 1e-4


def test_weighted_mean_weights_match_reference():
    import os
    from conftest import make_options
    from omega_b200 import priors
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "priorw_pet_mini.npz"))
    o = make_options("pet_mini")
    o.Ndx = o.Ndy = o.Ndz = 1
    assert np.array_equal(priors.weighted_mean_weights(o), f["wmean_111"])


def test_weighted_mean_user_weights_keep_their_sum():
    """Weights given in options.weighted_weights are passed as given, with
    their sum beside them: Weighted_mean (priors.h:103) divides them by
    af::sum of the weights for the means and uses them raw in the sums of
    types 4-6."""
    from conftest import make_options
    from omega_b200 import priors
    o = make_options("pet_mini")
    o.Ndx = o.Ndy = o.Ndz = 1
    w = np.arange(1, 28, dtype=np.float32)
    o.weighted_weights = w
    assert np.array_equal(priors.weighted_mean_weights(o), w)
    o.weighted_weights = np.zeros(27, np.float32)
    with pytest.raises(ValueError, match="sum to 0"):
        priors.weighted_mean_weights(o)


def test_wmean46_oracle_follows_the_reference_steps():
    """The types 4-6 restatement against the reference's ArrayFire steps
    written out literally (priors.h:125-210): pad by twice the window
    (symmetric, functions.hpp:216-260), convolve the padded image with the
    normalised weights (zero outside, same size), crop to the image grown by
    the window, then sum w_d g over the shifted means."""
    from scipy import ndimage
    rng = np.random.default_rng(3)
    shape = (9, 8, 7)
    nx, ny, nz = shape
    u = rng.uniform(0.2, 1.5, nx * ny * nz)
    w = rng.uniform(0.1, 1.0, 27)
    for mt in (4, 5, 6):
        ours = io.wmean_gradient46(u, shape, (1, 1, 1), w, mt, 1.0)
        U = u.reshape(shape, order='F')
        padd = np.pad(U, 2, mode='symmetric')
        W = w.reshape((3, 3, 3), order='F')
        f = {4: lambda a: a, 5: lambda a: 1 / a, 6: np.log}[mt]
        fi = {4: lambda a: a, 5: lambda a: 1 / a, 6: np.exp}[mt]
        M = fi(ndimage.convolve(f(padd), W / W.sum(), mode='constant', cval=0.0))[1:nx + 3, 1:ny + 3, 1:nz + 3]
        g = np.zeros_like(U)
        ut = np.maximum(U, 1e-6)
        for ll in range(3):
            for kk in range(3):
                for hh in range(3):
                    Md = M[hh:hh + nx, kk:kk + ny, ll:ll + nz]
                    if mt == 4:
                        t = np.log(np.maximum(U / Md, 1e-6))
                    elif mt == 5:
                        t = (ut - Md) / ut - ((ut - Md) / (np.sqrt(2) * ut)) ** 2
                    else:
                        t = 1 - Md / ut
                    g += W[hh, kk, ll] * t
        assert np.abs(g.ravel(order='F') - ours).max() < 1e-12 * np.abs(ours).max()


@pytest.mark.parametrize("flag", ["L", "FMH"])
def test_l_filter_and_fmh_count_as_priors(flag):
    """The L-filter and FMH are priors of the MAP algorithms: one of them
    with a second prior is refused before any launch, as any two priors are,
    and so is a window the reference's offsets grid does not follow."""
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.SinM = np.ones(int(o.Ndist) * int(o.Nang) * int(o.NSinos), np.float32)
    o.OSL_OSEM = True
    setattr(o, flag, True)
    o.MRP = True
    with pytest.raises(ValueError, match="needs one prior"):
        rec.reconstructions_main(o)


def test_proxtv_entry_points_validate_arguments():
    from omega_b200 import _native
    L = _native.lib()
    p = ctypes.c_void_p(16)
    f = ctypes.c_float
    assert L.omb_proxtv_dual(p, p, 8, 8, 4, f(0.5), f(0.0), 1, 0, None) != 0
    assert "beta" in L.omb_last_error().decode()
    assert L.omb_proxtv_dual(p, p, 8, 8, 4, f(0.5), f(0.1), 1, 2, None) != 0
    assert L.omb_proxtv_divergence(p, p, 8, 8, 4, 3, None) != 0
    assert "diff_type" in L.omb_last_error().decode()


def test_proxtv_needs_pdhg():
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.SinM = np.ones(int(o.Ndist) * int(o.Nang) * int(o.NSinos), np.float32)
    o.OSEM = True
    o.ProxTV = True
    with pytest.raises(ValueError, match="built for PDHG"):
        rec.reconstructions_main(o)


def test_proxtgv_entry_point_validates_arguments():
    from omega_b200 import _native
    L = _native.lib()
    p = ctypes.c_void_p(16)
    f = ctypes.c_float
    assert L.omb_proxtgv_step(p, p, p, p, p, 8, 8, 4, f(0.5), f(0.0), f(0.1), f(1.0), f(0.01), 1, 1, None) != 0
    assert "alpha0" in L.omb_last_error().decode()
    assert L.omb_proxtgv_step(p, p, p, p, None, 8, 8, 4, f(0.5), f(0.1), f(0.1), f(1.0), f(0.01), 1, 1, None) != 0
    assert "NULL" in L.omb_last_error().decode()


@pytest.mark.parametrize("case,match", [
    ("osem", "built for PDHG"), ("alpha", "alpha0TGV"), ("difftype", "forward differences"),
    ("both", "Select one")])
def test_tgv_option_checks(case, match):
    """options.TGV: PDHG only, positive balls, forward differences (the
    reference's backward-difference TGV kernels do not compile), one TV
    form at a time; all raised before the projector is set up."""
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.SinM = np.ones(int(o.Ndist) * int(o.Nang) * int(o.NSinos), np.float32)
    o.TGV = True
    o.alpha0TGV, o.alpha1TGV = 1.0, 1.0
    if case == "osem":
        o.OSEM = True
    else:
        o.PDHG = True
    if case == "alpha":
        o.alpha1TGV = 0.0
    if case == "difftype":
        o.derivativeType = 1
    if case == "both":
        o.ProxTV = True
    with pytest.raises(ValueError, match=match):
        rec.reconstructions_main(o)


def test_wmean46_rejects_windows_beyond_one_mirror():
    from omega_b200 import _native
    L = _native.lib()
    p = ctypes.c_void_p(16)
    f = ctypes.c_float
    assert L.omb_wmean_gradient(p, p, 8, 8, 3, 1, 1, 2, p, f(1.0), 4, f(1e-8), f(0.1), 0, None) != 0
    assert "twice the window" in L.omb_last_error().decode()
    assert L.omb_wmean_gradient(p, p, 8, 8, 3, 1, 1, 1, p, f(1.0), 7, f(1e-8), f(0.1), 0, None) != 0


def test_weighted_mean_single_slice_needs_flat_window():
    """One slice: the reference takes its 2-D path (no z window), so a z
    window is rejected before any launch."""
    from omega_b200 import _native
    st = _native.lib().omb_wmean_gradient(ctypes.c_void_p(16), ctypes.c_void_p(16), 8, 8, 1, 1, 1, 1,
                                          ctypes.c_void_p(16), ctypes.c_float(1.0), 1, ctypes.c_float(1e-8),
                                          ctypes.c_float(0.1), 0, None)
    assert st != 0
    assert "single slice" in _native.lib().omb_last_error().decode()


def _tv_golden():
    import os
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tv_anat.npz"))


class _TVOpts:
    Nx, Ny, Nz = 7, 6, 5
    TVsmoothing = 1e-3
    SATVPhi = 0.4
    C = 0.7
    eta = 0.02
    APLSsmoothing = 1e-4
    TV_use_anatomical = False
    TVtype = 1


def test_tv_setup_matches_reference_prepass():
    """The anatomical TV preparation equals the reference's own TVPrepass
    output bit for bit (tests/golden/tv_anat.npz): the min-max normalised
    reference image and the TVtype-1 tensor for two T; the other TV settings
    pick the reference's kernel form (ProjectorClass.h:900-918) and scalars
    (functions.hpp:1096-1113)."""
    from omega_b200 import _native, priors
    f = _tv_golden()
    o = _TVOpts()
    assert priors.tv_setup(o)[0] == _native.OMB_TV_PLAIN
    o.TVtype = 4
    assert priors.tv_setup(o) == (_native.OMB_TV_SATV, pytest.approx(0.4), 0.0, pytest.approx(1e-3), None)
    o.TVtype = 6
    assert priors.tv_setup(o)[:2] == (_native.OMB_TV_W1, pytest.approx(0.4))
    o.TV_use_anatomical = True
    o.TV_referenceImage = f["ref"]
    assert priors.tv_setup(o)[0] == _native.OMB_TV_PLAIN   # TVtype 6 with a reference: the plain kernel
    for T in (0.3, 2.0):
        o.TVtype, o.T = 1, T
        v, _, _, _, s = priors.tv_setup(o)
        assert v == _native.OMB_TV_ANAT1 and np.array_equal(s, f["s_T" + str(T)])
    o.TVtype = 2
    v, _, c, _, r = priors.tv_setup(o)
    assert v == _native.OMB_TV_ANAT2 and c == pytest.approx(0.7) and np.array_equal(r, f["ref_norm"])
    o.TVtype = 5
    v, _, c, sm, r = priors.tv_setup(o)
    assert v == _native.OMB_TV_APLS and c == pytest.approx(0.02) and sm == pytest.approx(1e-3)
    assert np.array_equal(r, f["ref_norm"])
    # the APLS prior: the raw reference image, eta and APLSsmoothing
    o.APLS_ref_image = f["ref"]
    v, _, c, sm, r = priors.tv_setup(o, apls=True)
    assert v == _native.OMB_TV_APLS and sm == pytest.approx(1e-4)
    assert np.array_equal(r, f["ref"].ravel(order="F"))


def test_tv_setup_rejects_bad_reference_images():
    from omega_b200 import priors
    o = _TVOpts()
    o.TV_use_anatomical, o.TVtype = True, 2
    o.TV_referenceImage = np.ones(10, np.float32)
    with pytest.raises(ValueError, match="size of the image"):
        priors.tv_setup(o)
    o.TV_referenceImage = np.ones(7 * 6 * 5, np.float32)
    with pytest.raises(ValueError, match="constant"):
        priors.tv_setup(o)
    o.TV_referenceImage = _tv_golden()["ref"]
    o.TVtype = 1
    with pytest.raises(ValueError, match="options.T"):
        priors.tv_setup(o)


def test_tv_variant_entry_validates_arguments():
    from omega_b200 import _native
    L = _native.lib()
    p = ctypes.c_void_p(16)
    f = ctypes.c_float
    # anatomical variants need the reference; SATV a nonzero sigma; unknown variants are refused
    assert L.omb_tv_gradient_ex(p, p, 8, 8, 4, f(1), f(1e-3), _native.OMB_TV_ANAT2, f(1), f(1), None, None) != 0
    assert "reference" in L.omb_last_error().decode()
    assert L.omb_tv_gradient_ex(p, p, 8, 8, 4, f(1), f(1e-3), _native.OMB_TV_SATV, f(0), f(0), None, None) != 0
    assert "sigma" in L.omb_last_error().decode()
    assert L.omb_tv_gradient_ex(p, p, 8, 8, 4, f(1), f(1e-3), 9, f(1), f(0), None, None) != 0


_TV_VARIANTS = {"satv": "OMB_TV_SATV", "tvw1": "OMB_TV_W1", "anat1": "OMB_TV_ANAT1", "anat2": "OMB_TV_ANAT2",
                "apls": "OMB_TV_APLS"}


def _tv_variant_inputs(variant, shape, seed, wide=False):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    u = rng.uniform(0.2, 1.0, n).astype(np.float32)
    if wide:
        # an iterate's range: zeros beside values up to 25
        u = (25.0 * u * (rng.uniform(0, 1, n) > 0.2)).astype(np.float32)
    ref = rng.uniform(0.0, 1.0, n).astype(np.float32)
    if variant == "anat1":
        from omega_b200 import priors
        S = priors.tv_anatomical_tensor(ref, *shape, 0.5)
    elif variant == "apls":
        S = 0.5 * ref     # keeps |d|^2 - (r . d)^2 + smooth positive
    elif variant == "anat2":
        S = ref
    else:
        S = None
    sigma, C = 0.3, (0.4 if variant == "anat2" else 0.05)
    return u, S, sigma, C


@pytest.mark.gpu
@pytest.mark.parametrize("wide", [False, True])
@pytest.mark.parametrize("variant", list(_TV_VARIANTS))
def test_tv_variant_kernels_match_oracle(cuda, variant, wide):
    """omb_tv_gradient_ex against the FP64 restatement of the TVKernel forms
    (pinned to the reference's kernel by test_refcl_pin), accumulating into
    an existing gradient."""
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    u, S, sigma, C = _tv_variant_inputs(variant, SHAPE, 61, wide)
    n = u.size
    U = torch.tensor(u, device=cuda)
    R = torch.tensor(S, device=cuda) if S is not None else None
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_tv_gradient_ex", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE,
                 0.8, 1e-3, getattr(_native, _TV_VARIANTS[variant]), sigma, C,
                 ctypes.c_void_p(R.data_ptr() if R is not None else 0), _stream(cuda))
    want = io.tv_gradient_variant(u.astype(np.float64), SHAPE, variant, 1e-3, 0.8, sigma=sigma, C=C,
                                  S=None if S is None else S.astype(np.float64))
    got = out.cpu().numpy() - 0.5
    assert orc.rel_l2(got, want) < 1e-5, (orc.rel_l2(got, want), np.abs(got - want).max(), np.abs(want).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["satv", "tvw1", "anat1", "anat2", "anat5", "apls_prior"])
def test_builtin_osl_osem_tv_variants(cuda, case):
    """One-step-late OSEM with each TV setting through the built-in entry,
    against the FP64 OSEM with the restated gradient."""
    from conftest import make_options
    from omega_b200 import priors
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    shape = (g.nx, g.ny, g.nz)
    rng = np.random.default_rng(71)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    truth = rng.uniform(0.5, 2.0, g.n_img)
    y = rng.poisson(orc.forward(orc.Geometry(full), truth, 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.OSL_OSEM = True
    o.TVsmoothing = 1e-2
    # small enough that sens + beta dTV stays away from 0 in every reached
    # voxel (at 2e-3 FP32 rounding alone moves the result by 5e-5); the
    # weighted TV's backward-z term (its w3.y weighting) reaches 100 times
    # the plain gradient, so it takes a tenth of that
    beta = 2e-5 if case == "tvw1" else 2e-4
    o.beta = beta
    o.Niter = 2
    ref_img = (truth + rng.uniform(0, 0.3, g.n_img)).astype(np.float32)
    if case == "apls_prior":
        o.APLS = True
        o.APLS_ref_image = 0.02 * ref_img
        o.APLSsmoothing = 1e-2
        o.eta = 0.1
    else:
        o.TV = True
        o.SATVPhi = 0.5
        if case in ("satv", "tvw1"):
            o.TVtype = 4 if case == "satv" else 6
        else:
            o.TV_use_anatomical = True
            o.TV_referenceImage = ref_img
            if case == "anat5":
                # APLS reads the raw (normalised) reference values into
                # sqrt(|d|^2 - (r . d)^2 + smooth), as TVKernel does: values
                # up to 0.3 keep it real; the maximum sits in voxel 0, which
                # is no voxel's forward neighbour
                ref5 = 0.3 * rng.uniform(0.0, 1.0, g.n_img).astype(np.float32)
                ref5[0] = 1.0
                o.TV_referenceImage = ref5
            o.TVtype = {"anat1": 1, "anat2": 2, "anat5": 5}[case]
            o.T, o.C, o.eta = 0.5, 0.3, 0.05
    variant, sigma, C, smooth, S = priors.tv_setup(o, apls=case == "apls_prior")
    name = {1: "satv", 2: "tvw1", 3: "anat1", 4: "anat2", 5: "apls"}[int(variant)]
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    S64 = None if S is None else S.astype(np.float64)

    def grad(v):
        return io.tv_gradient_variant(v, shape, name, smooth, beta, sigma=sigma, C=C, S=S64)
    want = orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=grad)
    x = out.ravel(order='F')
    assert np.all(np.isfinite(x))
    assert orc.rel_l2(x, want) < 5e-5, orc.rel_l2(x, want)
    # the variant reached the kernel: the plain TV gives another image
    plain = orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=lambda v: orc.tv_gradient(v, shape, smooth, beta))
    assert orc.rel_l2(x, plain) > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("mean_type", [4, 5, 6])
def test_weighted_mean_types_4_to_6(cuda, mean_type):
    """Kernel = restatement (weights not summing to 1), then BSREM with the
    prior through the built-in entry = the FP64 loop."""
    import torch
    from conftest import make_options
    from omega_b200 import _native, priors
    from omega_b200 import reconstruction as rec
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(30 + mean_type)
    n = int(np.prod(SHAPE))
    u = rng.uniform(0.3, 1.7, n).astype(np.float32)
    w = rng.uniform(0.05, 0.3, 27).astype(np.float32)
    U, W = torch.tensor(u, device=cuda), torch.tensor(w, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_wmean_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE,
                 1, 1, 1, ctypes.c_void_p(W.data_ptr()), float(np.sum(w, dtype=np.float32)), mean_type, 1e-8, 0.3, 0,
                 _stream(cuda))
    want = io.wmean_gradient46(u.astype(np.float64), SHAPE, (1, 1, 1), w.astype(np.float64), mean_type, 0.3)
    got = out.cpu().numpy() - 0.5
    assert orc.rel_l2(got, want) < 1e-5, orc.rel_l2(got, want)
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.BSREM = True
    o.weighted_mean = True
    o.mean_type = mean_type
    o.beta = 0.01
    o.Niter = 2
    lam = np.array([0.2, 0.12], np.float32)
    o.lambdaN = lam
    res, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    ww = priors.weighted_mean_weights(o).astype(np.float64)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam,
                      prior_grad=lambda v: io.wmean_gradient46(v, shape, (1, 1, 1), ww, mean_type, 0.01))
    x = res.ravel(order='F')
    assert np.all(np.isfinite(x))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("mean_type,no_norm", [(1, False), (2, False), (3, True)])
def test_weighted_mean(cuda, mean_type, no_norm):
    import torch
    from conftest import make_options
    from omega_b200 import _native, priors
    from omega_b200 import reconstruction as rec
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(20 + mean_type)
    n = int(np.prod(SHAPE))
    u = rng.uniform(0.5, 1.5, n).astype(np.float32)
    w = rng.uniform(0.01, 0.1, 27).astype(np.float32)
    U, W = torch.tensor(u, device=cuda), torch.tensor(w, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_wmean_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE,
                 1, 1, 1, ctypes.c_void_p(W.data_ptr()), float(w.sum()), mean_type, 1e-8, 0.3,
                 1 if no_norm else 0, _stream(cuda))
    want = 0.5 + io.wmean_gradient(u.astype(np.float64), SHAPE, (1, 1, 1), w.astype(np.float64) / float(w.sum()),
                                   mean_type, 0.3, 1e-8, no_norm)
    assert orc.rel_l2(out.cpu().numpy() - 0.5, want - 0.5) < 1e-5
    # BSREM with the prior: its MAP step keeps the image >= epps, so the
    # harmonic and geometric means stay finite where no ray reaches (one-step-
    # late OSEM drives those voxels to 0); the harmonic mean is left to the
    # kernel check above
    if mean_type == 2:
        return
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.BSREM = True
    o.weighted_mean = True
    o.mean_type = mean_type
    o.med_no_norm = no_norm
    o.beta = 0.01
    o.Niter = 2
    lam = np.array([0.2, 0.12], np.float32)
    o.lambdaN = lam
    res, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    ww = priors.weighted_mean_weights(o).astype(np.float64)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam,
                      prior_grad=lambda v: io.wmean_gradient(v, shape, (1, 1, 1), ww, mean_type, 0.01, g.epps,
                                                             no_norm))
    x = res.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)


def test_ramp_filters_match_reference():
    """omega_b200.filters.ramp_filter = the reference's rampFilt bit for bit
    (tests/golden/ramp_filters.npz: every window, two cut-offs, even and odd
    lengths), and the row filter's taps reproduce the Fourier-domain
    filtering of the reference (filtering / filteringInverse)."""
    import os
    from omega_b200 import filters
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ramp_filters.npz"))
    for k in g.files:
        if k.startswith("use2D"):
            continue
        w, c, N = k.rsplit("_", 2)
        ours = filters.ramp_filter(int(N), w, float(c), 0.25)
        assert ours.dtype == g[k].dtype and np.array_equal(ours, g[k]), k
    nf, f0, ff, h, hinv = filters.pdhg_row_filters(100, 0.7, "hann")
    assert nf == 128 and f0[0] == np.float32(1e-6)
    rng = np.random.default_rng(2)
    v = rng.normal(size=100 * 5)
    cols = v.reshape(-1, 100)
    for taps, filt, inv in ((h, f0, False), (hinv, ff, True)):
        direct = np.array([[np.dot(taps.astype(np.float64)[(i - np.arange(100)) % nf], col) for i in range(100)]
                           for col in cols]).ravel()
        fft = orc.row_filter_fft(v, 100, nf, filt, inverse=inv)
        assert np.abs(direct - fft).max() < 1e-7 * np.abs(fft).max()


def test_image_filter_is_the_separable_2d_ramp():
    """filters.image_filter_2d: F = f f^T / max (rampFilt.m:65-69), f the
    reference's 1-D rampFilt; its taps' separable circular convolution equals
    the Fourier-domain filtering2D; and the reference's Python use2D filter
    (tests/golden/ramp_filters.npz) is (N^2, N^2) with zeros in the N^2 values
    the library reads, which is why the 2-D filter is formed here."""
    import os
    from omega_b200 import filters
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ramp_filters.npz"))
    for N in (16, 32):
        assert tuple(g[f"use2D_shape_{N}"]) == (N * N, N * N)
        assert not np.any(g[f"use2D_first_{N}"])
    nf, F, h = filters.image_filter_2d(23, "hann", 0.9)
    assert nf == 32 and F.shape == (32, 32) and F.dtype == np.float32
    f = filters.ramp_filter(32, "hann", 0.9, 0.25)
    ff = np.outer(f, f).astype(np.float32)
    assert np.array_equal(F, ff / ff.max())
    shape = (23, 19, 3)
    rng = np.random.default_rng(4)
    v = rng.normal(size=int(np.prod(shape)))
    V = v.reshape(shape, order='F')
    hd = h.astype(np.float64)
    i = np.arange(23)
    j = np.arange(19)
    Kx = hd[(i[:, None] - i[None, :]) % nf]
    Ky = hd[(j[:, None] - j[None, :]) % nf]
    direct = np.einsum('ia,jb,abz->ijz', Kx, Ky, V).ravel(order='F')
    fft = orc.image_filter_fft(v, shape, nf, F)
    assert np.abs(direct - fft).max() < 1e-6 * np.abs(fft).max()


def test_filtered_relaxation_schedule():
    """lambdaFiltered until sub-iteration K, lambdaN from K on; K = 0 never
    switches; a switch inside an iteration needs equal values there."""
    from omega_b200.reconstruction import _filtered_relaxation

    class O:
        Niter = 4
        lambdaN = np.array([1., .5, .25, .125], np.float32)
        lambdaFiltered = np.array([9., 8., 7., 6.], np.float32)
    lam = O.lambdaN.copy()
    assert np.array_equal(_filtered_relaxation(O, lam, 4, 2), [9., 8., .25, .125])
    assert np.array_equal(_filtered_relaxation(O, lam, 0, 2), [9., 8., 7., 6.])
    assert np.array_equal(_filtered_relaxation(O, lam, 8, 2), [9., 8., 7., 6.])
    with pytest.raises(ValueError, match="multiple of subsets"):
        _filtered_relaxation(O, lam, 3, 2)
    O.lambdaFiltered = np.empty(0, np.float32)
    assert np.array_equal(_filtered_relaxation(O, lam, 3, 2), lam)


def test_pdhg_preconditioner_selection_is_checked():
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("ct_mini5")
    o.SinM = np.ones(int(o.nRowsD) * int(o.nColsD) * int(o.nProjections), np.float32)
    o.PDHG = True
    o.TV = True
    o.precondTypeImage = np.array([1, 0, 0, 0, 0, 0, 0], bool)
    with pytest.raises(ValueError, match="not PDHG"):
        rec.reconstructions_mainCT(o)


def test_ad_restatement_properties():
    """The AD restatement (ArrayFire's anisotropicDiffusion is not in the
    reference tree, so this prior's parity is unpinned): constants stay
    fixed, slices diffuse independently, a step agrees with the scheme
    written out for one voxel, and the smoothing lowers the spread."""
    shape = (9, 8, 3)
    rng = np.random.default_rng(11)
    n = int(np.prod(shape))
    assert np.abs(io.ad_smooth(np.full(n, 3.0), shape, 0.2, 0.7, 4) - 3.0).max() == 0.0
    u = rng.uniform(0.5, 1.5, n)
    U = u.reshape(shape, order='F')
    for mcde in (False, True):
        for expf in (True, False):
            a = io.ad_smooth(u, shape, 0.1, 0.6, 2, expf, mcde).reshape(shape, order='F')
            # slice 1 alone gives the same slice
            one = io.ad_smooth(U[:, :, 1:2].ravel(order='F'), (9, 8, 1), 0.1, 0.6, 2, expf, mcde)
            assert np.abs(one - a[:, :, 1].ravel(order='F')).max() < 1e-15
            assert a.std() < U.std()
    # one gradient-diffusion step at an interior voxel, written out
    i, j, k, dt, K = 4, 3, 1, 0.1, 0.6

    def c(g2):
        return np.exp(-g2 / K ** 2)
    V = U[:, :, k]
    C, E, W, S, N = V[i, j], V[i + 1, j], V[i - 1, j], V[i, j + 1], V[i, j - 1]
    SE, NE, SW, NW = V[i + 1, j + 1], V[i + 1, j - 1], V[i - 1, j + 1], V[i - 1, j - 1]
    gx_f = (E - C) ** 2 + ((S - N) / 2 + (SE - NE) / 2) ** 2 / 4
    gx_b = (C - W) ** 2 + ((S - N) / 2 + (SW - NW) / 2) ** 2 / 4
    gy_f = (S - C) ** 2 + ((E - W) / 2 + (SE - SW) / 2) ** 2 / 4
    gy_b = (C - N) ** 2 + ((E - W) / 2 + (NE - NW) / 2) ** 2 / 4
    want = C + dt * (c(gx_f) * (E - C) - c(gx_b) * (C - W) + c(gy_f) * (S - C) - c(gy_b) * (C - N))
    got = io.ad_smooth(u, shape, dt, K, 1, True, False).reshape(shape, order='F')[i, j, k]
    assert abs(got - want) < 1e-14


def test_ad_entry_point_and_options_validate():
    from conftest import make_options
    from omega_b200 import _native
    from omega_b200 import reconstruction as rec
    L = _native.lib()
    p = ctypes.c_void_p(16)
    f = ctypes.c_float
    assert L.omb_ad_gradient(p, p, 8, 8, 2, f(0.1), f(1.0), 1, 3, 2, f(1e-8), f(0.1), 0, None) != 0
    assert "FluxType" in L.omb_last_error().decode()
    assert L.omb_ad_gradient(p, p, 8, 8, 2, f(0.1), f(0.0), 1, 1, 2, f(1e-8), f(0.1), 0, None) != 0
    assert "KAD" in L.omb_last_error().decode()
    o = make_options("pet_mini")
    o.SinM = np.ones(int(o.Ndist) * int(o.Nang) * int(o.NSinos), np.float32)
    o.OSL_OSEM = True
    o.AD = True
    o.NiterAD = 0
    with pytest.raises(ValueError, match="NiterAD"):
        rec.reconstructions_main(o)


@pytest.mark.gpu
@pytest.mark.parametrize("flux,diffusion,no_norm", [(1, 2, False), (2, 2, False), (1, 1, True), (2, 1, False)])
def test_ad_kernel_matches_restatement(cuda, flux, diffusion, no_norm):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(12)
    n = int(np.prod(SHAPE))
    u = rng.uniform(0.5, 1.5, n).astype(np.float32)
    U = torch.tensor(u, device=cuda)
    out = torch.full((n,), 0.5, device=cuda)
    _native.call("omb_ad_gradient", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *SHAPE, 0.15,
                 0.4, 3, flux, diffusion, 1e-8, 0.3, 1 if no_norm else 0, _stream(cuda))
    want = io.ad_gradient(u.astype(np.float64), SHAPE, 0.15, 0.4, 3, flux == 1, diffusion == 2, 1e-8, no_norm)
    assert orc.rel_l2(out.cpu().numpy() - 0.5, 0.3 * want) < 1e-5, orc.rel_l2(out.cpu().numpy() - 0.5, 0.3 * want)


@pytest.mark.gpu
@pytest.mark.parametrize("diffusion,beta", [(2, 0.005), (1, 0.05)])
def test_builtin_osl_osem_with_ad(cuda, diffusion, beta):
    """OSL-OSEM with the AD prior (exponential flux; modified curvature, the
    default, or gradient diffusion) through the built-in entry against the
    FP64 loop.  The modified-curvature form normalises each flux by its
    gradient, which turns FP32 rounding in near-flat parts of the image into
    O(1) changes of direction; one-step-late OSEM feeds them back, so with
    that form the comparison runs at a tenth of the weight (at 0.05 the two
    loops part by 6 %)."""
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(13)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.OSL_OSEM = True
    o.AD = True
    o.TimeStepAD, o.KAD, o.NiterAD, o.DiffusionType = 0.1, 0.5, 2, diffusion
    o.beta = beta
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    ref = orc.osem(g, ys, np.ones(g.n_img), 2,
                   prior_grad=lambda v: beta * io.ad_gradient(v, shape, 0.1, 0.5, 2, True, diffusion == 2, g.epps))
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    # against the same one-step-late loop with a zero prior: the prior moves the image by 2-8 %
    assert orc.rel_l2(ref, orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=lambda v: 0.0 * v)) > 1e-2
