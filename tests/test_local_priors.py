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


def test_weighted_mean_user_weights_are_normalised():
    """Weights given in options.weighted_weights are divided by their sum, as
    Weighted_mean (priors.h:103) divides by af::sum of the weights."""
    from conftest import make_options
    from omega_b200 import priors
    o = make_options("pet_mini")
    o.Ndx = o.Ndy = o.Ndz = 1
    w = np.arange(1, 28, dtype=np.float32)
    o.weighted_weights = w
    got = priors.weighted_mean_weights(o)
    assert abs(float(got.sum()) - 1.0) < 1e-6
    assert np.allclose(got, w / w.sum(), rtol=1e-6)
    o.weighted_weights = np.zeros(27, np.float32)
    with pytest.raises(ValueError, match="sum to 0"):
        priors.weighted_mean_weights(o)


def test_weighted_mean_single_slice_needs_flat_window():
    """One slice: the reference takes its 2-D path (no z window), so a z
    window is rejected before any launch."""
    from omega_b200 import _native
    st = _native.lib().omb_wmean_gradient(ctypes.c_void_p(16), ctypes.c_void_p(16), 8, 8, 1, 1, 1, 1,
                                          ctypes.c_void_p(16), ctypes.c_float(1.0), 1, ctypes.c_float(1e-8),
                                          ctypes.c_float(0.1), 0, None)
    assert st != 0
    assert "single slice" in _native.lib().omb_last_error().decode()


@pytest.mark.parametrize("attrs", [dict(TVtype=4), dict(TVtype=6), dict(TV_use_anatomical=True)])
def test_tv_variants_not_built_are_rejected(attrs):
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.SinM = np.ones(int(o.Ndist) * int(o.Nang) * int(o.NSinos), np.float32)
    o.OSL_OSEM = True
    o.TV = True
    for k, v in attrs.items():
        setattr(o, k, v)
    with pytest.raises(ValueError, match="TV"):
        rec.reconstructions_main(o)


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
