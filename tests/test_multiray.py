"""Multi-ray PET projection (n_rays_transaxial x n_rays_axial rays per LOR
spread over the crystal pitch): the FP64 oracle against the reference's own
CPU projector with nRays2D / nRays3D (CPU, projector_functions.h:440-461,
1441-1466, 2045-2058), and the CUDA kernels against the oracle (GPU)."""
import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

TOL = 1e-5


@pytest.mark.skipif(orc.ref_lib() is None, reason="reference CPU projector not built")
@pytest.mark.parametrize("name,rays", [("pet_mini", (3, 2)), ("pet_mini_tof", (2, 1)), ("pet_mini", (1, 3))])
def test_multiray_oracle_matches_reference(name, rays):
    o = make_options(name)
    g = orc.Geometry(o)
    g.nr_xy, g.nr_z = rays
    rng = np.random.default_rng(1)
    x = rng.uniform(0.5, 2.0, g.n_img)
    for s in (0, 1):
        fp = orc.forward(g, x, s)
        assert orc.rel_l2(fp, orc.ref_multiray(g, x, s, True)) < 1e-12
        y = rng.uniform(0.0, 2.0, g.rays(s) * g.nbins)
        bp, sens = orc.backward(g, y, s, sens=True)
        ref_bp, ref_s = orc.ref_multiray(g, y, s, False, sens=True)
        assert orc.rel_l2(bp, ref_bp) < 1e-12 and orc.rel_l2(sens, ref_s) < 1e-12
        # the rays matter: one ray per LOR differs by several per cent
        assert orc.rel_l2(orc.forward(orc.Geometry(o), x, s), fp) > 1e-2


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


@pytest.mark.gpu
@pytest.mark.parametrize("name,rays", [("pet_mini", (3, 2)), ("pet_mini_tof", (2, 2)), ("pet_stype1", (2, 1))])
def test_multiray_gpu_matches_oracle(cuda, name, rays):
    o = make_options(name)
    o.n_rays_transaxial, o.n_rays_axial = rays
    o.initProj()
    g = orc.Geometry(o)
    rng = np.random.default_rng(2)
    x = rng.uniform(0.5, 2.0, g.n_img)
    for s in range(g.n_subsets):
        fp = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        assert orc.rel_l2(fp, orc.forward(g, x, s)) < TOL, s
        y = rng.uniform(0.0, 2.0, g.rays(s) * g.nbins)
        bp, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref_bp, ref_s = orc.backward(g, y, s, sens=True)
        assert orc.rel_l2(bp.cpu().numpy(), ref_bp) < TOL, s
        assert orc.rel_l2(sens.cpu().numpy(), ref_s) < TOL, s


@pytest.mark.gpu
def test_multiray_with_corrections_and_limits(cuda):
    from omega_b200 import _native
    o = make_options("pet_mini")
    o.n_rays_transaxial, o.n_rays_axial = 2, 2
    rng = np.random.default_rng(3)
    o.attenuation_correction = 1
    o.vaimennus = (0.0096 * rng.uniform(0.5, 1.5, int(np.ravel(o.N)[0]))).astype(np.float32)
    o.initProj()
    g = orc.Geometry(o)
    g.mu = o.vaimennus.astype(np.float64)
    x = rng.uniform(0.5, 2.0, g.n_img)
    assert orc.rel_l2(o.forwardProject(_t(x, cuda), 1).cpu().numpy(), orc.forward(g, x, 1)) < TOL
    # one ray per LOR only: the fixed-point backprojection and projector type 4
    o64 = make_options("pet_mini")
    o64.n_rays_transaxial = 2
    o64.use_64bit_atomics = True
    o64.initProj()
    with pytest.raises(_native.NativeError):
        o64.backwardProject(_t(np.ones(o64.measurementCount(0)), cuda), 0)
    o4 = make_options("pet_mini4")
    o4.n_rays_transaxial = 2
    with pytest.raises(_native.NativeError):
        o4.initProj()
