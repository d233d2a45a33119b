"""Relaxed PET algorithms (ROSEM, RAMLA, BSREM, ROSEM-MAP): the relaxation
schedule of the host entry against the reference's prepass rule, properties
of the FP64 restatement, and the native loop (built-in and custom-loop
entries) against that restatement on the GPU."""
import ctypes

import numpy as np
import pytest

from conftest import make_options
from oracle import image_oracle as io
from oracle import oracle as orc


def _pet(name, seed, scale=200):
    o = make_options(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(seed)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    full = make_options(name)
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), truth, 0) * scale).astype(np.float32) / scale
    o.SinM = y.copy()
    return o, g


def _subset_measurements(o, g):
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    return [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]


def test_default_relaxation_matches_prepass_rule():
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.Niter = 45
    lam = rec.relaxation(o)
    assert lam.dtype == np.float32 and lam.size == 45
    want = np.array([1. / (i / 20. + 1.) for i in range(45)], dtype=np.float32)
    assert np.array_equal(lam, want)
    assert np.array_equal(orc.default_relaxation(45), want)
    # the examples' np.zeros(1) means "use the default"
    o.lambdaN = np.zeros(1, dtype=np.float32)
    assert np.array_equal(rec.relaxation(o), want)


def test_relaxation_user_values_short_and_long(capsys):
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.Niter = 3
    o.lambdaN = np.array([0.5, 0.25, 0.125, 0.1, 0.05], dtype=np.float32)
    assert np.array_equal(rec.relaxation(o), np.array([0.5, 0.25, 0.125], dtype=np.float32))
    assert 'Later values are ignored' in capsys.readouterr().out
    o.lambdaN = np.array([0.5], dtype=np.float32)
    assert np.array_equal(rec.relaxation(o), orc.default_relaxation(3))
    assert 'Computing custom relaxation values' in capsys.readouterr().out


def test_rosem_at_unit_relaxation_is_osem():
    # x + x / s (rhs - s) = x rhs / s: the EM step without its + epps on rhs.
    # One subset: a voxel that some subset misses (s clamped to epps, rhs 0)
    # would drop to x - x = 0 in ROSEM and keep its value in OSEM.
    o = make_options("pet_mini")
    o.subsets, o.subsetType = 1, 8
    o.addProjector()
    g = orc.Geometry(o)
    rng = np.random.default_rng(11)
    y = rng.poisson(orc.forward(g, rng.uniform(0.5, 2.0, g.n_img), 0) * 200) / 200
    x_r = orc.relaxed(g, [y], np.ones(g.n_img), 2, "ROSEM", lam=np.ones(2, np.float32))
    x_o = orc.osem(g, [y], np.ones(g.n_img), 2)
    seen = orc.backward(g, None, 0, sens=True)[1] > 0
    assert seen.sum() > g.n_img // 2
    assert orc.rel_l2(x_r[seen], x_o[seen]) < 1e-4
    assert np.max(np.abs(x_r[~seen])) < 1e-12


def test_relaxed_fixed_point_at_consistent_data():
    # noise-free data of x_true: the ratio is 1 (RAMLA: 0) and x_true stays
    # put where the (one) subset sees it; unseen voxels: ROSEM scales them by
    # 1 - lam (sens clamped to epps, rhs 0), RAMLA leaves them
    o = make_options("pet_mini")
    o.subsets, o.subsetType = 1, 8
    o.addProjector()
    g = orc.Geometry(o)
    rng = np.random.default_rng(12)
    x_true = rng.uniform(0.5, 2.0, g.n_img)
    seen = orc.backward(g, None, 0, sens=True)[1] > 0
    ys = [orc.forward(g, x_true, 0)]
    for kind in ("ROSEM", "RAMLA"):
        x = orc.relaxed(g, ys, x_true, 1, kind, lam=np.full(1, 0.2, np.float32))
        # y / (fp + epps): off 1 by epps / fp only
        assert orc.rel_l2(x[seen], x_true[seen]) < 2e-5, kind
        want = x_true[~seen] * (1 - float(np.float32(0.2)) if kind == "ROSEM" else 1.0)
        assert np.allclose(x[~seen], want, rtol=1e-9), kind


def test_map_step_restatement():
    # BSREM with a zero prior is RAMLA; a positive gradient lowers the image
    o, g = _pet("pet_mini", 13)
    ys = _subset_measurements(o, g)
    lam = np.array([0.2, 0.1], np.float32)
    a = orc.relaxed(g, ys, np.ones(g.n_img), 2, "RAMLA", lam=lam)
    b = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam, prior_grad=lambda x: np.zeros_like(x))
    assert np.array_equal(a, b)
    c = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam, prior_grad=lambda x: np.full_like(x, 0.5))
    assert np.all(c <= b + 1e-12) and np.all(c >= g.epps)


def _run_builtin(o, method, n_iter, lam=None, graph=True, **prior):
    from omega_b200 import reconstruction as rec
    setattr(o, method, True)
    o.Niter = n_iter
    o.use_graph = graph
    if lam is not None:
        o.lambdaN = np.asarray(lam, dtype=np.float32)
    for k, v in prior.items():
        setattr(o, k, v)
    out, _ = rec.reconstructions_main(o)
    return out.ravel(order='F')


# With lam = 1 a ROSEM sub-iteration sets every voxel its subset misses to
# x - x (sensitivity clamped to epps, backprojection 0): 0 in FP64, a float
# residue on the GPU (and in the reference's float32 code), which later
# sub-iterations that do see the voxel multiply up.  The multi-subset cases
# therefore run lam < 1; the default schedule (lam[0] = 1) runs on one subset.
_LAM = [0.5, 0.4, 0.3]


@pytest.mark.gpu
@pytest.mark.parametrize("name,graph", [("pet_mini", True), ("pet_mini", False), ("pet_mini_tof", True),
                                        ("pet_stype1", True)])
def test_builtin_rosem_matches_oracle(cuda, name, graph):
    o, g = _pet(name, 21)
    x = _run_builtin(o, "ROSEM", 3, lam=_LAM, graph=graph)
    ys = _subset_measurements(o, g)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, "ROSEM", lam=np.float32(_LAM))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    # the relaxation matters: lam = 1 is (nearly) OSEM, not this
    assert orc.rel_l2(ref, orc.osem(g, ys, np.ones(g.n_img), 3)) > 1e-3


@pytest.mark.gpu
def test_builtin_rosem_default_schedule_one_subset(cuda):
    o = make_options("pet_mini")
    o.subsets, o.subsetType = 1, 8
    o.addProjector()
    g = orc.Geometry(o)
    rng = np.random.default_rng(27)
    o.SinM = (rng.poisson(orc.forward(g, rng.uniform(0.5, 2.0, g.n_img), 0) * 200) / 200).astype(np.float32)
    x = _run_builtin(o, "ROSEM", 3)
    assert np.array_equal(o.lambdaN, orc.default_relaxation(3))
    ref = orc.relaxed(g, _subset_measurements(o, g), np.ones(g.n_img), 3, "ROSEM")
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name,graph", [("pet_mini", True), ("pet_mini", False), ("pet_mini_tof", True)])
def test_builtin_ramla_matches_oracle(cuda, name, graph):
    o, g = _pet(name, 22)
    lam = [0.2, 0.12, 0.08]
    x = _run_builtin(o, "RAMLA", 3, lam=lam, graph=graph)
    ref = orc.relaxed(g, _subset_measurements(o, g), np.ones(g.n_img), 3, "RAMLA", lam=np.float32(lam))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert np.all(x >= g.epps)


@pytest.mark.gpu
@pytest.mark.parametrize("images", [True, False])
def test_builtin_bsrem_rdp_matches_oracle(cuda, images):
    """BSREM with RDP; with options.useImages (the default) the prior's
    neighbours outside the image are the edge voxel, without it 0, as the
    reference's texture and buffer paths read them."""
    o, g = _pet("pet_mini", 23)
    lam = [0.2, 0.12, 0.08]
    x = _run_builtin(o, "BSREM", 3, lam=lam, RDP=True, RDP_gamma=2.0, beta=0.05, useImages=images)
    shape = (g.nx, g.ny, g.nz)
    ys = _subset_measurements(o, g)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, "BSREM", lam=np.float32(lam),
                      prior_grad=lambda v: io.rdp_gradient(v, shape, 2.0, 0.05, g.epps, clamp=images))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    plain = orc.relaxed(g, ys, np.ones(g.n_img), 3, "RAMLA", lam=np.float32(lam))
    assert orc.rel_l2(ref, plain) > 1e-3  # the prior changes the result


@pytest.mark.gpu
@pytest.mark.parametrize("prior", ["Quad", "Huber"])
def test_builtin_rosem_map_matches_oracle(cuda, prior):
    from omega_b200 import priors
    o, g = _pet("pet_mini", 24)
    x = _run_builtin(o, "ROSEM_MAP", 3, lam=_LAM, beta=0.05, huber_delta=0.05, **{prior: True})
    shape = (g.nx, g.ny, g.nz)
    win = priors.prior_window(priors.normalised_weights(priors.neighbourhood_weights(o)), 1, 1, 1)
    delta = 0.05 if prior == "Huber" else np.inf

    def grad(v):
        return 0.05 * np.clip(io.psf_convolve(v, shape, win, (1, 1, 1)), -delta, delta)
    ys = _subset_measurements(o, g)
    lam = np.float32(_LAM)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, "ROSEM_MAP", lam=lam, prior_grad=grad)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.relaxed(g, ys, np.ones(g.n_img), 3, "ROSEM", lam=lam)) > 1e-4


@pytest.mark.gpu
def test_custom_loop_entries_match_builtin(cuda):
    """omb_rosem_subset / omb_ramla_subset / omb_map_step issued by hand give
    the built-in loop's image."""
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _ptr, _stream
    o, g = _pet("pet_mini", 25)
    lam = np.array([0.2, 0.12], np.float32)
    built = _run_builtin(o, "BSREM", 2, lam=lam, RDP=True, RDP_gamma=2.0, beta=0.05)
    dev = torch.device("cuda", o._device)
    st = _stream(dev)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [torch.from_numpy(np.ascontiguousarray(o.subsetMeasurements(m, s), dtype=np.float32)).to(dev)
          for s in range(g.n_subsets)]
    x = torch.ones(g.n_img, device=dev)
    wm = torch.empty(max(int(v.numel()) for v in ys), device=dev)
    wi = torch.empty(g.n_img, device=dev)
    du = torch.empty(g.n_img, device=dev)
    for it in range(2):
        for s in range(g.n_subsets):
            _native.call("omb_ramla_subset", o._handle, s, _ptr(x), _ptr(ys[s]), float(lam[it]), 1, _ptr(wm),
                         _ptr(wi), st)
        du.zero_()
        # the built-in loop clamps the prior's neighbours to the edge (options.useImages, the default)
        _native.call("omb_rdp_gradient_ex", _ptr(x), _ptr(du), g.nx, g.ny, g.nz, 2.0, float(g.epps), 0.05, 1, st)
        _native.call("omb_map_step", _ptr(x), _ptr(du), ctypes.c_int64(g.n_img), float(lam[it]), float(g.epps), st)
    assert orc.rel_l2(x.cpu().numpy(), built) < 1e-6
    # ROSEM sub-iterations by hand against the built-in ROSEM
    o2, _ = _pet("pet_mini", 25)
    built_r = _run_builtin(o2, "ROSEM", 1, lam=[0.7])
    sens = [torch.empty(g.n_img, device=dev) for _ in range(g.n_subsets)]
    for s in range(g.n_subsets):
        _native.call("omb_sensitivity", o2._handle, s, _ptr(sens[s]), st)
    x = torch.ones(g.n_img, device=dev)
    for s in range(g.n_subsets):
        _native.call("omb_rosem_subset", o2._handle, s, _ptr(x), _ptr(ys[s]), _ptr(sens[s]), 0.7, _ptr(wm),
                     _ptr(wi), st)
    assert orc.rel_l2(x.cpu().numpy(), built_r) < 1e-6


@pytest.mark.gpu
def test_relaxed_rejects_ct_and_missing_prior(cuda):
    from omega_b200 import reconstruction as rec
    o, _ = _pet("pet_mini", 26)
    o.BSREM = True
    with pytest.raises(ValueError, match="needs one prior"):
        rec.reconstructions_main(o)
    o.BSREM, o.RAMLA, o.OSEM = False, True, True
    with pytest.raises(ValueError, match="Select one"):
        rec.reconstructions_main(o)


def test_default_momentum_matches_prepass_rule(capsys):
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o.Niter = 3
    a = rec.momentum(o)
    S = int(o.subsets)
    want = np.zeros(3 * S, dtype=np.float32)
    oo = 0
    for kk in range(3):
        for ll in range(S):
            want[oo] = 1. + (0.45 * (kk * S + ll)) / (kk * S + ll + 100.)
            oo += 1
    assert np.array_equal(a, want) and np.array_equal(orc.default_momentum(3, S), want)
    assert 'Computing custom alpha values' in capsys.readouterr().out
    o.alpha_PKMA = np.linspace(1.0, 1.2, 3 * S + 2).astype(np.float32)
    assert np.array_equal(rec.momentum(o), o.alpha_PKMA[:3 * S])
    assert 'final values will be ignored' in capsys.readouterr().out


def test_pkma_and_mramla_restatement_properties():
    o, g = _pet("pet_mini", 31)
    ys = _subset_measurements(o, g)
    lam = np.array([0.3], np.float32)
    # alpha = 1: PKMA is the projected gradient step x - lam A^T(1 - y / fp)
    x1 = orc.relaxed(g, ys, np.ones(g.n_img), 1, "PKMA", lam=lam, alpha=np.ones(g.n_subsets, np.float32))
    assert np.all(x1 >= g.epps)
    # MRAMLA = PKMA at alpha = 1 with the gradient negated (before the bounds)
    x2 = orc.relaxed(g, ys, np.ones(g.n_img), 1, "MRAMLA", lam=lam)
    assert orc.rel_l2(x1, x2) < 1e-12
    # the upper bound: values at or above U land at U - epps
    x3 = orc.relaxed(g, ys, np.ones(g.n_img), 1, "MRAMLA", lam=np.array([5.0], np.float32), upper=1.5)
    assert np.max(x3) <= 1.5 and np.any(x3 == 1.5 - g.epps)
    # MBSREM with a zero prior is MRAMLA
    x4 = orc.relaxed(g, ys, np.ones(g.n_img), 1, "MBSREM", lam=lam, prior_grad=lambda v: np.zeros_like(v))
    assert np.array_equal(x4, x2)


@pytest.mark.gpu
@pytest.mark.parametrize("name,graph", [("pet_mini", True), ("pet_mini", False), ("pet_mini_tof", True)])
def test_builtin_pkma_matches_oracle(cuda, name, graph):
    o, g = _pet(name, 32)
    lam = [0.3, 0.2, 0.15]
    x = _run_builtin(o, "PKMA", 3, lam=lam, graph=graph)
    ref = orc.relaxed(g, _subset_measurements(o, g), np.ones(g.n_img), 3, "PKMA", lam=np.float32(lam))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert np.array_equal(o.alpha_PKMA, orc.default_momentum(3, g.n_subsets))


@pytest.mark.gpu
def test_builtin_pkma_with_rdp_matches_oracle(cuda):
    o, g = _pet("pet_mini", 33)
    lam = [0.3, 0.2, 0.15]
    x = _run_builtin(o, "PKMA", 3, lam=lam, RDP=True, RDP_gamma=2.0, beta=0.05)
    shape = (g.nx, g.ny, g.nz)
    ys = _subset_measurements(o, g)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, "PKMA", lam=np.float32(lam),
                      prior_grad=lambda v: io.rdp_gradient(v, shape, 2.0, 0.05, g.epps, clamp=True))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.relaxed(g, ys, np.ones(g.n_img), 3, "PKMA", lam=np.float32(lam))) > 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("upper", [0.0, 1.6])
def test_builtin_mramla_matches_oracle(cuda, upper):
    o, g = _pet("pet_mini", 34)
    lam = [0.2, 0.12, 0.08]
    o.U = upper
    x = _run_builtin(o, "MRAMLA", 3, lam=lam)
    ref = orc.relaxed(g, _subset_measurements(o, g), np.ones(g.n_img), 3, "MRAMLA", lam=np.float32(lam),
                      upper=upper if upper > 0 else 10000.0)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    if upper > 0:
        assert np.max(x) < upper


@pytest.mark.gpu
def test_builtin_mbsrem_quad_matches_oracle(cuda):
    from omega_b200 import priors
    o, g = _pet("pet_mini", 35)
    lam = [0.2, 0.12, 0.08]
    x = _run_builtin(o, "MBSREM", 3, lam=lam, Quad=True, beta=0.05)
    shape = (g.nx, g.ny, g.nz)
    win = priors.prior_window(priors.normalised_weights(priors.neighbourhood_weights(o)), 1, 1, 1)

    def grad(v):
        return 0.05 * io.psf_convolve(v, shape, win, (1, 1, 1))
    ys = _subset_measurements(o, g)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, "MBSREM", lam=np.float32(lam), prior_grad=grad)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.relaxed(g, ys, np.ones(g.n_img), 3, "MRAMLA", lam=np.float32(lam))) > 1e-4


@pytest.mark.gpu
def test_pkma_mbsrem_entries_match_builtin(cuda):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _ptr, _stream
    o, g = _pet("pet_mini", 36)
    lam = np.array([0.3, 0.2], np.float32)
    built = _run_builtin(o, "PKMA", 2, lam=lam)
    alpha = orc.default_momentum(2, g.n_subsets)
    dev = torch.device("cuda", o._device)
    st = _stream(dev)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [torch.from_numpy(np.ascontiguousarray(o.subsetMeasurements(m, s), dtype=np.float32)).to(dev)
          for s in range(g.n_subsets)]
    x = torch.ones(g.n_img, device=dev)
    wm = torch.empty(max(int(v.numel()) for v in ys), device=dev)
    wi = torch.empty(g.n_img, device=dev)
    for it in range(2):
        for s in range(g.n_subsets):
            _native.call("omb_pkma_subset", o._handle, s, _ptr(x), _ptr(ys[s]), float(lam[it]),
                         float(alpha[it * g.n_subsets + s]), None, 1, None, 0, _ptr(wm), _ptr(wi), st)
    assert orc.rel_l2(x.cpu().numpy(), built) < 1e-6
    o2, _ = _pet("pet_mini", 36)
    built2 = _run_builtin(o2, "MRAMLA", 1, lam=[0.2])
    x = torch.ones(g.n_img, device=dev)
    for s in range(g.n_subsets):
        _native.call("omb_mbsrem_subset", o2._handle, s, _ptr(x), _ptr(ys[s]), 0.2, 10000.0, None, 1, None, 0,
                     _ptr(wm), _ptr(wi), st)
    assert orc.rel_l2(x.cpu().numpy(), built2) < 1e-6


@pytest.mark.gpu
def test_precond_image_matches_oracle(cuda):
    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _ptr, _stream
    o, g = _pet("pet_mini", 40)
    o.initProj()
    dev = torch.device("cuda", o._device)
    d = torch.empty(g.n_img, device=dev)
    w = torch.empty(g.n_img, device=dev)
    _native.call("omb_precond_image", o._handle, _ptr(d), _ptr(w), _stream(dev))
    ref = orc.precond_image(g)
    assert np.any(ref == 1.0)      # voxels no ray crosses
    assert orc.rel_l2(d.cpu().numpy(), ref) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("method,mode", [("PKMA", 1), ("PKMA", 2), ("MRAMLA", 2), ("MBSREM", 1)])
def test_builtin_preconditioned_matches_oracle(cuda, method, mode):
    o, g = _pet("pet_mini", 41)
    lam = [0.6, 0.4, 0.3] if mode == 2 else [0.3, 0.2, 0.15]
    o.precondTypeImage = np.array([mode == 1, mode == 2, False, False, False, False, False])
    extra = {"RDP": True, "RDP_gamma": 2.0, "beta": 0.05} if method == "MBSREM" else {}
    x = _run_builtin(o, method, 3, lam=lam, **extra)
    shape = (g.nx, g.ny, g.nz)
    grad = (lambda v: io.rdp_gradient(v, shape, 2.0, 0.05, g.epps, clamp=True)) if method == "MBSREM" else None
    ys = _subset_measurements(o, g)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, method, lam=np.float32(lam), prior_grad=grad, precond=mode)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    plain = orc.relaxed(g, ys, np.ones(g.n_img), 3, method, lam=np.float32(lam), prior_grad=grad)
    assert orc.rel_l2(ref, plain) > 1e-3


def _other_precond_case(case, g, rng):
    """(options, oracle keyword arguments, method, relaxation) of one of the
    other preconditioners; the relaxation keeps each run well-conditioned."""
    S = g.n_subsets
    n_iter = 3
    if case == "type2":
        ref = rng.uniform(0.5, 1.5, g.n_img).astype(np.float32)
        return (dict(precondTypeImage=np.array([0, 0, 1, 0, 0, 0, 0], bool), referenceImage=ref),
                dict(precond=3, ref=ref.astype(np.float64)), "PKMA", [0.6, 0.4, 0.3])
    if case == "type3":
        a = rng.uniform(0.5, 1.0, n_iter * S).astype(np.float32)
        return (dict(precondTypeImage=np.array([0, 0, 0, 1, 0, 0, 0], bool), alphaPrecond=a),
                dict(alpha_precond=a), "PKMA", [0.3, 0.2, 0.15])
    if case == "type4":
        return (dict(precondTypeImage=np.array([0, 0, 0, 0, 1, 0, 0], bool), gradV1=0.5, gradV2=2.5, gradInitIter=2,
                     gradLastIter=5, derivativeType=2),
                dict(grad_precond=dict(v1=0.5, v2=2.5, init=2, last=5, diff_type=2)), "PKMA", [0.3, 0.2, 0.15])
    if case == "type0+4":
        return (dict(precondTypeImage=np.array([1, 0, 0, 0, 1, 0, 0], bool), gradInitIter=1, gradLastIter=1,
                     derivativeType=0),
                dict(precond=1, grad_precond=dict(v1=0.5, v2=2.5, init=1, last=1, diff_type=0)), "MRAMLA",
                [0.3, 0.2, 0.15])
    if case == "type6":
        return (dict(precondTypeImage=np.array([0, 0, 0, 0, 0, 0, 1], bool), U=5.0),
                dict(curv_precond=True, upper=5.0), "MRAMLA", [0.02, 0.012, 0.008])
    if case == "meas0":
        return (dict(precondTypeMeas=np.array([1, 0], bool)), dict(meas_precond=True), "PKMA", [0.3, 0.2, 0.15])
    if case == "relax":
        return (dict(computeRelaxationParameters=True, relaxationScaling=True),
                dict(auto_relax=True, relax_scaling=True), "PKMA", [0.3, 0.2, 0.15])
    if case in ("type5", "type5k0", "type5mramla"):
        # the filtering-based image preconditioner: one filtered iteration with its own relaxation, or
        # (K = 0) the first sub-iteration only with lambdaFiltered = lambdaN throughout
        from omega_b200 import filters
        nf, F, _ = filters.image_filter_2d(g.nx, "hann")
        K = 0 if case == "type5k0" else S
        lf = None if case == "type5k0" else np.array([0.05, 0.04, 0.03], np.float32)
        opts = dict(precondTypeImage=np.array([0, 0, 0, 0, 0, 1, 0], bool), filteringIterations=K, filterWindow="hann")
        if lf is not None:
            opts["lambdaFiltered"] = lf
        return (opts, dict(img_filter=dict(nf=nf, F=F, K=K), lam_filtered=lf),
                "MRAMLA" if case == "type5mramla" else "PKMA", [0.3, 0.2, 0.15])
    raise KeyError(case)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["type2", "type3", "type4", "type0+4", "type6", "meas0", "relax", "type5", "type5k0",
                                  "type5mramla"])
def test_builtin_other_preconditioners(cuda, case):
    """Image preconditioners 2, 3, 4, 5 and 6, the measurement preconditioner
    0 and PKMA's automatic relaxation through the built-in entry against the
    FP64 loop; each changes the result."""
    o, g = _pet("pet_mini", 42)
    rng = np.random.default_rng(43)
    opts, kw, method, lam = _other_precond_case(case, g, rng)
    x = _run_builtin(o, method, 3, lam=lam, **opts)
    ys = _subset_measurements(o, g)
    upper = kw.pop("upper", 10000.0)
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 3, method, lam=np.float32(lam), upper=upper, **kw)
    assert np.all(np.isfinite(x))
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    plain = orc.relaxed(g, ys, np.ones(g.n_img), 3, method, lam=np.float32(lam), upper=upper)
    assert orc.rel_l2(ref, plain) > 1e-3


def test_other_preconditioners_validate():
    """Rejected selections raise before any device work."""
    o, g = _pet("pet_mini", 44)
    from omega_b200 import reconstruction as rec
    o.PKMA = True
    o.precondTypeImage = np.array([0, 0, 0, 0, 0, 1, 0], bool)
    o.filteringIterations = 3
    o.Niter = 2
    o.lambdaN = np.array([1., .5], np.float32)
    o.lambdaFiltered = np.array([.3, .2], np.float32)
    with pytest.raises(ValueError, match="multiple of subsets"):
        rec.reconstructions_main(o)
    nx = int(np.ravel(o.Nx)[0])
    o.Ny = 2 * nx + 1
    with pytest.raises(ValueError, match="Ny <="):
        rec.reconstructions_main(o)
    o.Ny = nx
    o.precondTypeImage = np.array([1, 1, 0, 0, 0, 0, 0], bool)
    with pytest.raises(ValueError, match="Only one"):
        rec.reconstructions_main(o)
    o.precondTypeImage = np.zeros(7, bool)
    o.precondTypeMeas = np.array([0, 1], bool)
    with pytest.raises(ValueError, match="measurement preconditioner"):
        rec.reconstructions_main(o)
