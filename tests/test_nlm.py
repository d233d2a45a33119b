"""Non-local priors (NLM, NLTV, NLM-MRP, NLRD, NL Lange, MRP + Lange,
NLGGMRF): the restatement (oracle/image_oracle.py) pinned against the
reference's CPU function NLMFunc (oracle/_ref) in its CPU variant, the patch
weights against the reference's NLMPrepass (tests/golden/nlm_gauss.npz), the
CUDA kernel against the restatement, and OSL-OSEM with the NLM prior."""
import ctypes
import os

import numpy as np
import pytest

from oracle import image_oracle as io
from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPE = (14, 13, 11)
CASES = [((1, 1, 1), (1, 1, 1)), ((2, 2, 1), (1, 1, 0))]


def _gauss(pw, sd=2.0):
    class O:
        pass
    o = O()
    o.Nlx, o.Nly, o.Nlz = pw
    o.NLM_gauss = sd
    from omega_b200 import priors
    return priors.nlm_gaussian(o)


def _ref_nlm(u, ref, g, sw, pw, h, t, gamma, pqc, anat):
    L = orc.ref_lib()
    P = ctypes.POINTER(ctypes.c_double)
    i32, u32, d = ctypes.c_int32, ctypes.c_uint32, ctypes.c_double
    L.ref_nlm_d.argtypes = [P, P, P, P, i32, i32, i32, i32, i32, i32, u32, u32, u32, d, i32, d, d, d, d, d, i32]
    grad = np.zeros(u.size)
    gd = np.asarray(g, dtype=np.float64)
    L.ref_nlm_d(grad.ctypes.data_as(P), ref.ctypes.data_as(P), u.ctypes.data_as(P), gd.ctypes.data_as(P), *sw, *pw,
                *SHAPE, h, t, gamma, 1e-8, *pqc, 1 if anat else 0)
    return grad


def test_patch_weights_match_reference():
    f = np.load(os.path.join(HERE, "golden", "nlm_gauss.npz"))
    assert np.array_equal(_gauss((1, 1, 1), 2.0), f["g_111"])
    assert np.array_equal(_gauss((2, 2, 1), 1.5), f["g_221"])


@pytest.mark.parametrize("sw,pw", CASES)
def test_cpu_variant_matches_reference(sw, pw):
    if orc.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(0)
    u = rng.uniform(0.5, 1.5, int(np.prod(SHAPE)))
    ref = rng.uniform(0.5, 1.5, u.size)
    g = _gauss(pw)
    for t in range(7):
        for anat in (False, True):
            want = _ref_nlm(u, ref, g, sw, pw, 0.05, t, 2.0, (2.0, 1.5, 0.01), anat)
            got = io.nlm_gradient(u, SHAPE, g, sw, pw, 0.05, 1e-8, t, gamma=2.0, ggmrf=(2.0, 1.5, 0.01),
                                  u_ref=ref if anat else None, cpu_mode=True)
            assert np.count_nonzero(want) > 0
            assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want)), (t, anat)


def test_kernel_variant_differs_only_in_epps_placement_and_borders():
    # interior voxels: W = epps + sum w against 1 / (sum w + epps) -- equal to rounding
    rng = np.random.default_rng(1)
    u = rng.uniform(0.5, 1.5, int(np.prod(SHAPE)))
    g = _gauss((1, 1, 1))
    a = io.nlm_gradient(u, SHAPE, g, (1, 1, 1), (1, 1, 1), 0.05, 1e-8, 0)
    b = io.nlm_gradient(u, SHAPE, g, (1, 1, 1), (1, 1, 1), 0.05, 1e-8, 0, cpu_mode=True)
    inner = b != 0
    assert np.max(np.abs(a[inner] - b[inner])) < 1e-12
    assert np.count_nonzero(a[~inner]) > 0   # the kernel also covers the border


def test_flat_image_has_zero_gradient():
    u = np.full(int(np.prod(SHAPE)), 2.0)
    g = _gauss((1, 1, 1))
    for t in (0, 1, 3, 4, 6):
        assert np.max(np.abs(io.nlm_gradient(u, SHAPE, g, (1, 1, 1), (1, 1, 1), 0.05, 1e-8, t,
                                             ggmrf=(2.0, 1.5, 0.01)))) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("sw,pw", CASES)
def test_kernel_matches_restatement(cuda, sw, pw):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    rng = np.random.default_rng(2)
    n = int(np.prod(SHAPE))
    u = rng.uniform(0.5, 1.5, n)
    ref = rng.uniform(0.5, 1.5, n)
    g = _gauss(pw)
    U = torch.tensor(u, dtype=torch.float32, device=cuda)
    R = torch.tensor(ref, dtype=torch.float32, device=cuda)
    G = torch.tensor(g, dtype=torch.float32, device=cuda)
    S = (ctypes.c_int32 * 3)(*sw)
    Pw = (ctypes.c_int32 * 3)(*pw)
    pqc = (ctypes.c_float * 3)(2.0, 1.5, 0.01)
    for t in range(7):
        for anat in (False, True):
            out = torch.full((n,), 0.25, device=cuda)
            adaptive = anat and t == 0   # the adaptive weighting once, with the reference image
            _native.call("omb_nlm_gradient", ctypes.c_void_p(U.data_ptr()),
                         ctypes.c_void_p(R.data_ptr()) if anat else None, ctypes.c_void_p(out.data_ptr()),
                         *SHAPE, S, Pw, ctypes.c_void_p(G.data_ptr()), 0.05, 1e-8, 0.7, t, 2.0, pqc,
                         1 if adaptive else 0, 0.02, _stream(cuda))
            want = 0.25 + 0.7 * io.nlm_gradient(u.astype(np.float32), SHAPE, g, sw, pw, 0.05, 1e-8, t, gamma=2.0,
                                                ggmrf=(2.0, 1.5, 0.01),
                                                u_ref=ref.astype(np.float32) if anat else None,
                                                adaptive_s=0.02 if adaptive else None)
            got = out.cpu().numpy()
            assert orc.rel_l2(got - 0.25, want - 0.25) < 2e-5, (t, anat, orc.rel_l2(got - 0.25, want - 0.25))


@pytest.mark.gpu
def test_builtin_osl_osem_with_nlm(cuda):
    from conftest import make_options
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(6)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.OSL_OSEM = True
    o.NLM = True
    o.NLMsigma = 0.3
    o.beta = 0.002
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    gw = np.asarray(o.gaussianNLM, dtype=np.float64)
    sw = (int(o.Ndx), int(o.Ndy), int(o.Ndz))

    def grad(v):
        return 0.002 * io.nlm_gradient(v, shape, gw, sw, (1, 1, 1), 0.09, g.epps, 0)
    ref = orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=grad)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.osem(g, ys, np.ones(g.n_img), 2)) > 1e-4
