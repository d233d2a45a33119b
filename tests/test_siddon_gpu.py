"""Parity of the CUDA improved-Siddon projector (projector type 1) with the
FP64 oracle and the reference's own CPU projector fixtures.

Bar: relative L2 <= 1e-5 in FP32 for projections and images; the int64
fixed-point backprojection is bit-identical run to run.
"""
import numpy as np
import pytest

from conftest import load_golden, make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _init(name, **attrs):
    """Options with attribute overrides applied before addProjector()."""
    from configs import CONFIGS, apply
    from make_golden import CONFIGS_EXTRA
    from omega_b200.projector import proj
    base = CONFIGS[name] if name in CONFIGS else CONFIGS_EXTRA[name]
    o = apply(proj.projectorClass(), dict(base, **attrs))
    o.addProjector()
    o.initProj()
    return o


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


CASES = ["pet_mini", "pet_tof_small", "pet_mini_tof", "pet_odd_span1", "ct_mini", "pet_stype1", "pet_stype2",
         "pet_stype4", "pet_stype5"]


@pytest.mark.parametrize("name", CASES)
def test_forward_matches_oracle(cuda, name):
    o = _init(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(7)
    x = rng.uniform(0.1, 2.0, g.n_img).astype(np.float32)
    for s in range(g.n_subsets):
        y = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        ref = orc.forward(g, x, s)
        assert y.shape == ref.shape
        assert orc.rel_l2(y, ref) < TOL, (name, s, orc.rel_l2(y, ref))


@pytest.mark.parametrize("name", CASES)
def test_backward_and_sensitivity_match_oracle(cuda, name):
    o = _init(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(8)
    for s in range(g.n_subsets):
        y = rng.uniform(0.0, 3.0, g.rays(s) * g.nbins).astype(np.float32)
        img, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref, rsens = orc.backward(g, y, s, sens=True)
        assert orc.rel_l2(img.cpu().numpy(), ref) < TOL, (name, s)
        assert orc.rel_l2(sens.cpu().numpy(), rsens) < TOL, (name, s)


@pytest.mark.parametrize("name", ["pet_mini", "pet_tof_small"])
def test_against_reference_cpu_fixtures(cuda, name):
    """Same inputs as the reference's own OpenMP projector run in the fixtures."""
    o = _init(name)
    p = load_golden("proj", name)
    for k in [k for k in p if k.startswith("fp_")]:
        y = o.forwardProject(_t(p["image"], cuda), int(k[3:])).cpu().numpy()
        assert orc.rel_l2(y, p[k]) < TOL, k
    img, sens = o.backwardProject(_t(p["bp_in_0"], cuda), 0, sens=True)
    assert orc.rel_l2(img.cpu().numpy(), p["bp_0"]) < TOL
    assert orc.rel_l2(sens.cpu().numpy(), p["sens_0"]) < TOL


def test_cfg0_all_subsets(cuda):
    """The CPU-runnable PET workload (144 x 144 x 31, 8 subsets) end to end."""
    o = _init("pet_cfg0")
    g = orc.Geometry(o)
    rng = np.random.default_rng(9)
    x = rng.uniform(0.5, 1.5, g.n_img).astype(np.float32)
    for s in range(g.n_subsets):
        y = o.forwardProject(_t(x, cuda), s)
        assert orc.rel_l2(y.cpu().numpy(), orc.forward(g, x, s)) < TOL
        bp = o.backwardProject(y, s)
        assert orc.rel_l2(bp.cpu().numpy(), orc.backward(g, y.cpu().numpy(), s)) < TOL


def test_operator_sugar(cuda):
    o = _init("pet_mini")
    rng = np.random.default_rng(1)
    x = _t(rng.random(int(o.N[0])), cuda)
    o.subset = 2
    y1 = o * x
    y2 = o.forwardProject(x, 2)
    assert np.array_equal(y1.cpu().numpy(), y2.cpu().numpy())
    b1 = o.T() * y1
    assert not o.trans
    b2 = o.backwardProject(y1, 2)
    assert orc.rel_l2(b1.cpu().numpy(), b2.cpu().numpy()) < 1e-6


def test_adjoint_on_gpu(cuda):
    o = _init("pet_mini_tof")
    rng = np.random.default_rng(2)
    x = rng.random(int(o.N[0])).astype(np.float32)
    m = o.measurementCount(1)
    y = rng.random(m).astype(np.float32)
    a = float(np.dot(o.forwardProject(_t(x, cuda), 1).cpu().numpy().astype(np.float64), y))
    b = float(np.dot(x.astype(np.float64), o.backwardProject(_t(y, cuda), 1).cpu().numpy()))
    assert abs(a - b) < 1e-5 * abs(a)


@pytest.mark.parametrize("name", ["pet_mini", "pet_tof_small"])
def test_fixed64_bit_identical_run_to_run(cuda, name):
    o = _init(name, use_64bit_atomics=True)
    g = orc.Geometry(o)
    rng = np.random.default_rng(4)
    y = _t(rng.uniform(0, 2, g.rays(0) * g.nbins), cuda)
    a, sa = o.backwardProject(y, 0, sens=True)
    b, sb = o.backwardProject(y, 0, sens=True)
    assert np.array_equal(a.cpu().numpy().view(np.uint32), b.cpu().numpy().view(np.uint32))
    assert np.array_equal(sa.cpu().numpy().view(np.uint32), sb.cpu().numpy().view(np.uint32))
    ref, rs = orc.backward(g, y.cpu().numpy(), 0, sens=True)
    assert orc.rel_l2(a.cpu().numpy(), ref) < TOL
    assert orc.rel_l2(sa.cpu().numpy(), rs) < TOL


def test_frames_batch_equals_single_frames(cuda):
    """The multi-frame launch (one walk per ray for up to 8 frames) equals
    frame-by-frame projections."""
    import ctypes
    import torch
    from omega_b200 import _native
    o = _init("pet_mini")
    n = int(o.N[0])
    m = o.measurementCount(-1)
    rng = np.random.default_rng(6)
    for nf in (1, 3, 5, 11):
        imgs = _t(rng.random((nf, n)), cuda)
        ys = torch.empty((nf, m), device=cuda)
        st = torch.cuda.current_stream().cuda_stream
        _native.call("omb_forward_frames", o._handle, -1, nf, ctypes.c_void_p(imgs.data_ptr()), n,
                     ctypes.c_void_p(ys.data_ptr()), m, ctypes.c_void_p(st))
        back = torch.empty((nf, n), device=cuda)
        _native.call("omb_backward_frames", o._handle, -1, nf, ctypes.c_void_p(ys.data_ptr()), m,
                     ctypes.c_void_p(back.data_ptr()), n, ctypes.c_void_p(st))
        for f in range(nf):
            y1 = torch.empty(m, device=cuda)
            _native.call("omb_forward", o._handle, -1, ctypes.c_void_p(imgs[f].data_ptr()),
                         ctypes.c_void_p(y1.data_ptr()), ctypes.c_void_p(st))
            assert torch.equal(y1, ys[f])
            ref = torch.zeros(n, device=cuda)
            _native.call("omb_backward", o._handle, -1, ctypes.c_void_p(ys[f].data_ptr()),
                         ctypes.c_void_p(ref.data_ptr()), None, 0, ctypes.c_void_p(st))
            assert orc.rel_l2(back[f].cpu().numpy(), ref.cpu().numpy()) < 1e-6


def test_zero_measurements_give_zero_image(cuda):
    o = _init("pet_mini")
    import torch
    y = torch.zeros(o.measurementCount(0), device=cuda)
    img = o.backwardProject(y, 0)
    assert float(img.abs().sum()) == 0.0


def test_bad_subset_raises(cuda):
    from omega_b200._native import NativeError
    o = _init("pet_mini")
    import torch
    with pytest.raises(NativeError, match="out of range"):
        o.forwardProject(torch.ones(int(o.N[0]), device=cuda), 9)
    with pytest.raises(ValueError, match="elements"):
        o.forwardProject(torch.ones(5, device=cuda), 0)


def test_osem_subset_step_matches_oracle(cuda):
    """One fused OSEM iteration (FP, ratio, BP, EM per subset) vs the oracle loop."""
    import ctypes
    import torch
    from omega_b200 import _native
    o = _init("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(12)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    ys = [rng.poisson(orc.forward(g, truth, s) * 20.0).astype(np.float32) for s in range(g.n_subsets)]
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = g.n_img
    x = torch.ones(n, device=cuda)
    sens = [torch.empty(n, device=cuda) for _ in range(g.n_subsets)]
    for s in range(g.n_subsets):
        _native.call("omb_sensitivity", o._handle, s, ctypes.c_void_p(sens[s].data_ptr()), st)
    wm = torch.empty(max(o.measurementCount(s) for s in range(g.n_subsets)), device=cuda)
    wi = torch.empty(n, device=cuda)
    yd = [_t(y, cuda) for y in ys]
    for s in range(g.n_subsets):
        _native.call("omb_osem_subset", o._handle, s, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(yd[s].data_ptr()),
                     ctypes.c_void_p(sens[s].data_ptr()), ctypes.c_void_p(wm.data_ptr()),
                     ctypes.c_void_p(wi.data_ptr()), st)
    ref = orc.osem(g, ys, np.ones(n), 1)
    assert orc.rel_l2(x.cpu().numpy(), ref) < 2e-5


def test_loglik_matches_oracle(cuda):
    import ctypes
    import torch
    from omega_b200 import _native
    rng = np.random.default_rng(3)
    n = 1_000_003
    y = rng.poisson(3.0, n).astype(np.float32)
    fp = rng.uniform(0.0, 6.0, n).astype(np.float32)
    L = _native.lib()
    work = torch.empty(int(L.omb_reduce_workspace_bytes(n)) // 8 + 1, dtype=torch.float64, device=cuda)
    out = ctypes.c_double()
    yd, fd = _t(y, cuda), _t(fp, cuda)
    _native.call("omb_loglik", ctypes.c_void_p(yd.data_ptr()), ctypes.c_void_p(fd.data_ptr()), n,
                 ctypes.c_float(1e-5), ctypes.byref(out), ctypes.c_void_p(work.data_ptr()),
                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    ref = orc.loglik(y, fp, np.float32(1e-5))
    assert abs(out.value - ref) <= 1e-9 * abs(ref)


def test_intersection_count_matches_oracle(cuda):
    import ctypes
    import torch
    from omega_b200 import _native
    o = _init("pet_mini")
    g = orc.Geometry(o)
    n = ctypes.c_int64()
    _native.call("omb_intersection_count", o._handle, 1, ctypes.byref(n),
                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    ref = orc.intersections(g, 1)
    assert abs(n.value - ref) <= 1e-4 * ref


@pytest.mark.parametrize("name", ["pet_mini", "pet_stype1", "pet_stype4", "pet_odd_span1"])
def test_system_matrix_backprojection(cuda, name):
    """Backprojections through the resident transposed system matrix
    (siddon_bp_matrix = 1) against the FP64 oracle and the ray-driven
    atomics, for every subset, frame batches of 1, 5 (4 + 1) and 11 (8 + 3)
    frames, and bit-identical call to call."""
    import ctypes

    import torch
    from omega_b200 import _native
    o = _init(name)
    g = orc.Geometry(o)
    n = int(o.N[0])
    rng = np.random.default_rng(7)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for s in range(g.n_subsets):
        m = o.measurementCount(s)
        for nf in (1, 5, 11):
            ys = _t(rng.uniform(0.0, 2.0, (nf, m)), cuda)
            outs = []
            for mat in (0, 1, 1):
                o.tuning = {"siddon_bp_matrix": mat}
                back = torch.empty((nf, n), device=cuda)
                _native.call("omb_backward_frames", o._handle, s, nf, ctypes.c_void_p(ys.data_ptr()), m,
                             ctypes.c_void_p(back.data_ptr()), n, st)
                outs.append(back.cpu().numpy())
            assert np.array_equal(outs[1].view(np.uint32), outs[2].view(np.uint32))
            for f in range(nf):
                assert orc.rel_l2(outs[1][f], outs[0][f]) < 1e-6, (s, nf, f)
            ref = orc.backward(g, ys[nf - 1].cpu().numpy().astype(np.float64), s)
            assert orc.rel_l2(outs[1][nf - 1], ref) < TOL


def test_system_matrix_backprojection_with_corrections(cuda):
    """Corrections set after a matrix was built replace it (the weights fold
    them in): the backprojection follows the new corrections."""
    import ctypes

    import torch
    from omega_b200 import _native
    o = _init("pet_mini")
    g = orc.Geometry(o)
    n = int(o.N[0])
    m = o.measurementCount(-1)
    rng = np.random.default_rng(8)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    y = _t(rng.uniform(0.0, 2.0, m), cuda)

    def bp(mat):
        o.tuning = {"siddon_bp_matrix": mat}
        b = torch.empty(n, device=cuda)
        _native.call("omb_backward", o._handle, -1, ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                     None, 0, st)
        return b.cpu().numpy()
    plain = bp(1)
    n_all = o.measurementCount(-1)
    w = rng.uniform(0.5, 1.5, n_all).astype(np.float32)
    _native.call("omb_set_corrections", o._handle, w.ctypes.data_as(ctypes.c_void_p), w.size, None, 0, None)
    corr = bp(1)
    assert orc.rel_l2(corr, bp(0)) < 1e-6
    assert orc.rel_l2(corr, plain) > 1e-3
