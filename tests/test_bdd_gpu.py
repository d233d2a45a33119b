"""Parity of the CUDA branchless distance-driven projector (type 5), the
PDHG+TV iteration and the power method with the FP64 oracle (the
reference's SAT formulation evaluated exactly).  Bar: relative L2 <= 1e-5."""
import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _init(name, **attrs):
    """Options with attribute overrides applied before addProjector()."""
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), dict(CONFIGS[name], **attrs))
    o.addProjector()
    o.initProj()
    return o


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _phantom(g, seed=0):
    rng = np.random.default_rng(seed)
    xs = (np.arange(g.nx) + 0.5) * g.d[0] + g.b[0]
    ys = (np.arange(g.ny) + 0.5) * g.d[1] + g.b[1]
    zs = (np.arange(g.nz) + 0.5) * g.d[2] + g.b[2]
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    img = 0.01 * ((X / 25.) ** 2 + (Y / 20.) ** 2 + (Z / 18.) ** 2 < 1)
    img = img + 0.02 * (((X - 5) / 6.) ** 2 + (Y / 8.) ** 2 + ((Z + 3) / 5.) ** 2 < 1)
    return (img + 0.002 * rng.random(img.shape)).ravel(order="F")


@pytest.mark.parametrize("subsets", [1, 4])
def test_bdd_forward_matches_oracle(cuda, subsets):
    o = _init("ct_mini5", subsets=subsets)
    g = orc.Geometry(o)
    x = _phantom(g)
    for s in range(g.n_subsets):
        y = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        ref = orc.bdd_forward(g, x, s)
        assert y.shape == ref.shape
        assert orc.rel_l2(y, ref) < TOL, (s, orc.rel_l2(y, ref))


@pytest.mark.parametrize("subsets", [1, 3])
def test_bdd_backward_matches_oracle(cuda, subsets):
    o = _init("ct_mini5", subsets=subsets)
    g = orc.Geometry(o)
    rng = np.random.default_rng(3)
    for s in range(g.n_subsets):
        y = rng.uniform(0.0, 2.0, g.rays(s)).astype(np.float32)
        img, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref, rs = orc.bdd_backward(g, y, s, sens=True)
        assert orc.rel_l2(img.cpu().numpy(), ref) < TOL, s
        assert orc.rel_l2(sens.cpu().numpy(), rs) < TOL, s


def test_bdd_random_image_forward(cuda):
    """Random voxel values (large local gradients) stress the footprint edges."""
    o = _init("ct_mini5")
    g = orc.Geometry(o)
    x = np.random.default_rng(5).uniform(0, 1, g.n_img)
    y = o.forwardProject(_t(x, cuda), 0).cpu().numpy()
    assert orc.rel_l2(y, orc.bdd_forward(g, x, 0)) < TOL


def test_power_method_matches_oracle(cuda):
    import torch
    from omega_b200 import reconstruction as rec
    o = _init("ct_mini5")
    g = orc.Geometry(o)
    L = rec.power_method(o, 20, seed=7)
    x0 = torch.randn(g.n_img, generator=torch.Generator().manual_seed(7)).abs().numpy()
    Lr = orc.power_method(g, 20, x0=x0)
    assert abs(L - Lr) < 1e-5 * Lr


def test_pdhg_tv_matches_oracle(cuda):
    from omega_b200 import reconstruction as rec
    o = _init("ct_mini5")
    g = orc.Geometry(o)
    truth = _phantom(g, 1)
    y = orc.bdd_forward(g, truth, -1)
    tau = 1.0 / orc.power_method(g, 10, seed=2)
    x0 = np.full(g.n_img, 1e-4)
    solver = rec.PDHG(o, y, beta=0.05, tv_smooth=1e-4, tau=tau, x0=x0)
    x = solver.iterate(4).cpu().numpy()
    ref = orc.pdhg_tv(g, y, x0, 4, tau, beta=0.05, smooth=1e-4, eps=float(o.epps))
    assert orc.rel_l2(x, ref) < TOL, orc.rel_l2(x, ref)


def test_pdhg_graph_replay_equals_eager(cuda):
    """The type-5 pair is a gather (no atomics): graph replays are bit-identical."""
    from omega_b200 import reconstruction as rec
    o = _init("ct_mini5")
    g = orc.Geometry(o)
    y = orc.bdd_forward(g, _phantom(g, 2), -1)
    a = rec.PDHG(o, y, beta=0.02, tau=1e-3).iterate(6, use_graph=False).cpu().numpy()
    b = rec.PDHG(o, y, beta=0.02, tau=1e-3).iterate(6, use_graph=True).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_pdhg_split_calls_equal_fused_iteration(cuda):
    """omb_forward -> omb_pdhg_dual -> omb_backward -> omb_pdhg_primal is the
    same computation as omb_pdhg_iteration, bit for bit."""
    import ctypes

    import torch
    from omega_b200 import _native
    o = _init("ct_mini5")
    g = orc.Geometry(o)
    y = _t(orc.bdd_forward(g, _phantom(g, 3), -1), cuda)
    n, m = g.n_img, g.rays(-1)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    runs = []
    for split in (False, True):
        x = torch.full((n,), 1e-3, device=cuda)
        xn, u, p = torch.empty_like(x), x.clone(), torch.zeros(m, device=cuda)
        wm, wi = torch.empty(m, device=cuda), torch.empty(n, device=cuda)
        for _ in range(3):
            if split:
                _native.call("omb_forward", o._handle, -1, P(x), P(wm), st)
                _native.call("omb_pdhg_dual", P(p), P(wm), P(y), m, 1.0, st)
                _native.call("omb_backward", o._handle, -1, P(p), P(wi), None, 0, st)
                _native.call("omb_pdhg_primal", o._handle, P(x), P(wi), P(u), P(xn), 1e-3, 1.0, 0.03, 1e-4, 1, st)
            else:
                _native.call("omb_pdhg_iteration", o._handle, P(x), P(xn), P(u), P(p), P(y), 1e-3, 1.0, 1.0, 0.03,
                             1e-4, 1, P(wm), P(wi), st)
            x, xn = xn, x
        runs.append(x.cpu().numpy())
    assert np.array_equal(runs[0].view(np.uint32), runs[1].view(np.uint32))


def test_osem_graph_replay_matches_eager(cuda):
    from omega_b200 import reconstruction as rec
    o = _init("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(4)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    m = np.concatenate([rng.poisson(orc.forward(g, truth, s) * 10.0) for s in range(g.n_subsets)]).astype(np.float32)
    a = rec.OSEM(o, m).iterate(3, use_graph=False).cpu().numpy()
    b = rec.OSEM(o, m).iterate(3, use_graph=True).cpu().numpy()
    assert orc.rel_l2(a, b) < 1e-6
    ys = [m[int(o.nTotMeas[s]):int(o.nTotMeas[s + 1])] for s in range(g.n_subsets)]
    ref = orc.osem(g, ys, np.ones(g.n_img), 3)
    assert orc.rel_l2(a, ref) < 5e-5


def test_osem_batch_equals_per_frame_osem(cuda):
    """omb_osem_subset_frames: three studies in one batch give each study's
    own OSEM result."""
    from omega_b200 import reconstruction as rec
    o = _init("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(8)
    ms = []
    for f in range(3):
        truth = rng.uniform(0.5, 2.0, g.n_img)
        ms.append(np.concatenate([rng.poisson(orc.forward(g, truth, s) * 10.0) for s in range(g.n_subsets)]))
    m = np.stack(ms).astype(np.float32)
    xb = rec.OSEMBatch(o, m).iterate(3, use_graph=True).cpu().numpy()
    for f in range(3):
        x1 = rec.OSEM(o, m[f]).iterate(3).cpu().numpy()
        assert orc.rel_l2(xb[f], x1) < 1e-6, f


@pytest.mark.parametrize("name,subsets", [("ct_mini5", 1), ("ct_mini5", 3), ("ct_fine5", 1)])
def test_bdd_ray_backward_matches_oracle(cuda, name, subsets):
    """The ray-driven scatter backprojection (OMB_BP_RAY) against the FP64
    adjoint of the forward projection, image and sensitivity."""
    o = _init(name, subsets=subsets)
    o.bddRayBackprojection = True
    g = orc.Geometry(o)
    rng = np.random.default_rng(41)
    for s in range(g.n_subsets):
        y = rng.uniform(0.0, 2.0, g.rays(s)).astype(np.float32)
        img, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref, rs = orc.bdd_backward_ray(g, y, s, sens=True)
        assert orc.rel_l2(img.cpu().numpy(), ref) < TOL, s
        assert orc.rel_l2(sens.cpu().numpy(), rs) < TOL, s


def test_bdd_ray_backward_is_adjoint_on_gpu(cuda):
    o = _init("ct_mini5")
    o.bddRayBackprojection = True
    g = orc.Geometry(o)
    rng = np.random.default_rng(42)
    x = rng.random(g.n_img).astype(np.float32)
    y = rng.random(g.rays(0)).astype(np.float32)
    a = float(np.dot(o.forwardProject(_t(x, cuda), 0).cpu().numpy().astype(np.float64), y))
    b = float(np.dot(x.astype(np.float64), o.backwardProject(_t(y, cuda), 0).cpu().numpy()))
    assert abs(a - b) < 1e-5 * abs(a)


def test_bdd_ray_backward_fixed64_bit_identical(cuda):
    """int64 fixed-point scatter (bddRayBackprojection = 'int64'):
    bit-identical run to run, and equal to the FP64 adjoint within the FP32
    bar."""
    o = _init("ct_mini5", bddRayBackprojection="int64")
    g = orc.Geometry(o)
    y = _t(np.random.default_rng(43).uniform(0.0, 2.0, g.rays(0)), cuda)
    a, sa = o.backwardProject(y, 0, sens=True)
    b, sb = o.backwardProject(y, 0, sens=True)
    assert np.array_equal(a.cpu().numpy().view(np.uint32), b.cpu().numpy().view(np.uint32))
    assert np.array_equal(sa.cpu().numpy().view(np.uint32), sb.cpu().numpy().view(np.uint32))
    ref, rs = orc.bdd_backward_ray(g, y.cpu().numpy(), 0, sens=True)
    assert orc.rel_l2(a.cpu().numpy(), ref) < TOL
    assert orc.rel_l2(sa.cpu().numpy(), rs) < TOL
