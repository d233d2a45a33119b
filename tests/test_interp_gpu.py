"""Parity of the CUDA interpolation projector (type 4) with the FP64 oracle:
PET forward/backward (with and without TOF, whole-sinogram and
measurement-level subsets), the int64 fixed-point backprojection (bit
identical run to run), and the CT forward and voxel-driven backward.
Bar: relative L2 <= 1e-5."""
import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _init(name, **attrs):
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), dict(CONFIGS[name], **attrs))
    o.addProjector()
    o.initProj()
    return o


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _image(g, seed):
    rng = np.random.default_rng(seed)
    xs = (np.arange(g.nx) + 0.5) * g.d[0] + g.b[0]
    ys = (np.arange(g.ny) + 0.5) * g.d[1] + g.b[1]
    zs = (np.arange(g.nz) + 0.5) * g.d[2] + g.b[2]
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    r = max(abs(g.b[0]), abs(g.b[1]))
    img = 1.0 + ((X / (0.6 * r)) ** 2 + (Y / (0.5 * r)) ** 2 < 1) + 0.5 * rng.random(X.shape)
    return img.ravel(order="F")


@pytest.mark.parametrize("name", ["pet_mini4", "pet_mini4_tof", "pet_half4", "ct_mini4"])
def test_interp_forward_matches_oracle(cuda, name):
    o = _init(name)
    g = orc.Geometry(o)
    x = _image(g, 1)
    for s in range(g.n_subsets):
        y = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        ref = orc.interp_forward(g, x, s)
        assert y.shape == ref.shape
        assert orc.rel_l2(y, ref) < TOL, (s, orc.rel_l2(y, ref))


@pytest.mark.parametrize("name", ["pet_mini4", "pet_mini4_tof", "pet_half4"])
def test_interp_pet_backward_matches_oracle(cuda, name):
    o = _init(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(2)
    for s in range(g.n_subsets):
        y = rng.uniform(0.0, 2.0, g.rays(s) * g.nbins)
        img, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref, rs = orc.interp_backward(g, y, s, sens=True)
        assert orc.rel_l2(img.cpu().numpy(), ref) < TOL, (s, orc.rel_l2(img.cpu().numpy(), ref))
        assert orc.rel_l2(sens.cpu().numpy(), rs) < TOL, s


def test_interp_fixed64_is_bit_reproducible(cuda):
    o = _init("pet_mini4_tof", use_64bit_atomics=True)
    g = orc.Geometry(o)
    y = np.random.default_rng(3).uniform(0.0, 2.0, g.rays(0) * g.nbins)
    a, sa = o.backwardProject(_t(y, cuda), 0, sens=True)
    b, sb = o.backwardProject(_t(y, cuda), 0, sens=True)
    a, b, sa, sb = (t.cpu().numpy() for t in (a, b, sa, sb))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(sa.view(np.uint32), sb.view(np.uint32))
    ref, rs = orc.interp_backward(g, y, 0, sens=True)
    assert orc.rel_l2(a, ref) < TOL and orc.rel_l2(sa, rs) < TOL


def test_interp_sensitivity_matches_oracle(cuda):
    import ctypes

    import torch
    from omega_b200 import _native
    o = _init("pet_mini4")
    g = orc.Geometry(o)
    sens = torch.empty(g.n_img, device=cuda)
    _native.call("omb_sensitivity", o._handle, 1, ctypes.c_void_p(sens.data_ptr()),
                 ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream))
    ref = np.maximum(orc.interp_backward(g, None, 1), float(o.epps))
    assert orc.rel_l2(sens.cpu().numpy(), ref) < TOL


def test_interp_ct_backward_matches_oracle(cuda):
    o = _init("ct_mini4")
    g = orc.Geometry(o)
    rng = np.random.default_rng(4)
    for s in range(g.n_subsets):
        y = rng.uniform(0.0, 2.0, g.rays(s))
        img, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref, rs = orc.interp_ct_backward(g, y, s, sens=True)
        assert orc.rel_l2(img.cpu().numpy(), ref) < TOL, (s, orc.rel_l2(img.cpu().numpy(), ref))
        assert orc.rel_l2(sens.cpu().numpy(), rs) < TOL, s


def test_interp_osem_matches_oracle(cuda):
    from omega_b200 import reconstruction as rec
    o = _init("pet_mini4")
    g = orc.Geometry(o)
    truth = _image(g, 5)
    m = np.concatenate([np.random.default_rng(6).poisson(orc.interp_forward(g, truth, s) * 20.0)
                        for s in range(g.n_subsets)]).astype(np.float32)
    x = rec.OSEM(o, m).iterate(2).cpu().numpy()
    ys = [m[int(o.nTotMeas[s]):int(o.nTotMeas[s + 1])] for s in range(g.n_subsets)]
    ref = orc.osem(g, ys, np.ones(g.n_img), 2, forward=orc.interp_forward,
                   backward=lambda gg, yy, ss, sens=False: orc.interp_backward(gg, yy, ss, sens=sens))
    assert orc.rel_l2(x, ref) < 5e-5


@pytest.mark.parametrize("name", ["pet_mini4", "pet_mini4_tof", "ct_mini4", "pet_mini"])
def test_bf16_image_reads_error_is_stated(cuda, name):
    """BF16 image reads (FP32 accumulation): the relative L2 error against the
    FP64 oracle stays below 4e-3 (BF16 keeps 8 significant bits; the sums
    average the per-voxel rounding) and is not zero (the BF16 path ran)."""
    o = _init(name, imageReadPrecision="bf16", maxFramesBF16=2)
    g = orc.Geometry(o)
    x = _image(g, 11)
    fwd = orc.interp_forward if int(o.projector_type) == 4 else orc.forward
    for s in range(g.n_subsets):
        y = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        err = orc.rel_l2(y, fwd(g, x, s))
        assert 1e-6 < err < 4e-3, (s, err)
