"""Projector types 2 (orthogonal distance) and 3 (volume of intersection) on
the GPU against the FP64 restatement of the same kernel (pinned to the
reference CPU projector by test_orth_oracle.py) at 1e-5 relative L2:
subsets, measurement-level subsets, TOF (type 3), corrections, list-mode
events, mixed projector pairs and the built-in OSEM."""
import warnings

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5
TUBES = {2: dict(tube_width_z=4.0, tube_width_xy=9.8), 3: dict(tube_radius=3.0)}


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _opts(base, pt, tube=None, **kw):
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    cfg = dict(CONFIGS[base], projector_type=pt)
    cfg.update(TUBES[tube or pt % 10 if pt % 10 in (2, 3) else pt // 10])
    cfg.update(kw)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        o = apply(proj.projectorClass(), cfg)
        o.addProjector()
    return o


def _check_subsets(o, g, cuda, rng, subsets=None):
    x = rng.uniform(0.5, 2.0, g.n_img)
    for s in (subsets if subsets is not None else range(g.n_subsets)):
        fp = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        ref = orc.orth_forward(g, x, s) if g.fp_type in (2, 3) else orc.forward(g, x, s)
        assert np.count_nonzero(ref) > 0
        assert orc.rel_l2(fp, ref) < TOL, (s, orc.rel_l2(fp, ref))
        y = rng.uniform(0.0, 2.0, g.rays(s) * g.nbins)
        bp, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        rb, rs = orc.orth_backward(g, y, s, sens=True) if g.bp_type in (2, 3) else orc.backward(g, y, s, sens=True)
        assert orc.rel_l2(bp.cpu().numpy(), rb) < TOL, (s, orc.rel_l2(bp.cpu().numpy(), rb))
        assert orc.rel_l2(sens.cpu().numpy(), rs) < TOL, s


@pytest.mark.parametrize("pt", [2, 3])
@pytest.mark.parametrize("base", ["pet_mini", "pet_stype1", "pet_odd_span1"])
def test_orth_matches_oracle(cuda, pt, base):
    o = _opts(base, pt)
    o.initProj()
    _check_subsets(o, orc.Geometry(o), cuda, np.random.default_rng(pt))


def test_volume_tof_matches_oracle(cuda):
    o = _opts("pet_mini_tof", 3)
    o.initProj()
    g = orc.Geometry(o)
    assert g.nbins == 7
    _check_subsets(o, g, cuda, np.random.default_rng(5), subsets=[0, 3])


@pytest.mark.parametrize("pt", [2, 3])
def test_orth_narrow_and_wide_tubes(cuda, pt):
    # a tube narrower than a voxel (the scans stop at the ray's own voxel) and
    # one several voxels wide; type 2 without the transaxial spread
    for kw in ({"tube_width_z": 2.0, "tube_width_xy": 0.0}, {"tube_width_z": 14.0}) if pt == 2 else \
            ({"tube_radius": 0.5}, {"tube_radius": 8.0}):
        o = _opts("pet_mini", pt, **kw)
        o.initProj()
        _check_subsets(o, orc.Geometry(o), cuda, np.random.default_rng(9), subsets=[1])


@pytest.mark.parametrize("pt", [2, 3])
def test_orth_with_corrections(cuda, pt):
    o = _opts("pet_mini", pt)
    rng = np.random.default_rng(11)
    total = int(np.ravel(o.nTotMeas)[-1])
    n_img = int(np.ravel(o.N)[0])
    o.normalization_correction = 1
    o.normalization = rng.uniform(0.5, 1.5, total).astype(np.float32)
    o.attenuation_correction = 1
    o.CTAttenuation = True
    o.vaimennus = (0.0096 * rng.uniform(0.5, 1.5, n_img)).astype(np.float32)
    o.initProj()
    g = orc.Geometry(o)
    g.w = o.normalization.astype(np.float64)
    g.mu = o.vaimennus.astype(np.float64)
    _check_subsets(o, g, cuda, rng, subsets=[0, 2])


def test_pairs_with_type4_backprojection_rejected(cuda):
    # the reference's set-up gives types 24 / 34 no type-4 sampling length
    # (coordinates.py:241 lists 42 and 43 only), so their backprojector has none
    from omega_b200 import _native
    for pt in (24, 34):
        o = _opts("pet_mini", pt, tube=pt // 10)
        with pytest.raises(_native.NativeError, match="sampling length"):
            o.initProj()


@pytest.mark.parametrize("pt", [12, 21, 13, 31, 42, 43])
def test_mixed_projector_pairs(cuda, pt):
    o = _opts("pet_mini", pt, tube=2 if 2 in (pt // 10, pt % 10) else 3)
    o.initProj()
    g = orc.Geometry(o)
    assert (g.fp_type, g.bp_type) == (pt // 10, pt % 10)
    if 4 in (g.fp_type, g.bp_type):
        # the type-4 half is checked by its own tests; here the orth half of the pair
        rng = np.random.default_rng(13)
        x = rng.uniform(0.5, 2.0, g.n_img)
        if g.fp_type in (2, 3):
            fp = o.forwardProject(_t(x, cuda), 0).cpu().numpy()
            assert orc.rel_l2(fp, orc.orth_forward(g, x, 0)) < TOL
        else:
            y = rng.uniform(0.0, 2.0, g.rays(0))
            bp = o.backwardProject(_t(y, cuda), 0).cpu().numpy()
            assert orc.rel_l2(bp, orc.orth_backward(g, y, 0)) < TOL
        return
    _check_subsets(o, g, cuda, np.random.default_rng(13), subsets=[0])


@pytest.mark.parametrize("pt", [2, 3])
def test_orth_listmode_events(cuda, pt):
    from conftest import make_listmode_options
    o = make_listmode_options("pet_mini", n_events=3000, event_seed=3, projector_type=pt, **TUBES[pt])
    o.initProj()
    g = orc.Geometry(o)
    assert g.modality == 2
    _check_subsets(o, g, cuda, np.random.default_rng(17))


@pytest.mark.parametrize("pt", [2, 3])
def test_builtin_osem_with_orth(cuda, pt):
    from omega_b200 import reconstruction as rec
    o = _opts("pet_mini", pt)
    g = orc.Geometry(o)
    rng = np.random.default_rng(19)
    full = _opts("pet_mini", pt, subsets=1, subsetType=8)
    y = rng.poisson(orc.orth_forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), -1) * 50) / 50
    o.SinM = y.astype(np.float32)
    o.OSEM = True
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    ref = orc.osem(g, ys, np.ones(g.n_img), 2, forward=orc.orth_forward, backward=orc.orth_backward)
    assert orc.rel_l2(out.ravel(order='F'), ref) < 5e-5, orc.rel_l2(out.ravel(order='F'), ref)


@pytest.mark.parametrize("pt", [2, 3])
def test_orth_system_matrix_backprojection(cuda, pt):
    """Types 2 / 3 (non-TOF) backprojected through the transposed system
    matrix of the tube weights (tuning siddon_bp_matrix = 1) against the
    ray-driven atomics and the FP64 oracle, for every subset and frame
    batches of 1, 5 and 11, bit-identical call to call."""
    import ctypes

    import torch
    from omega_b200 import _native
    o = _opts("pet_mini", pt)
    o.initProj()
    g = orc.Geometry(o)
    n = int(o.N[0])
    rng = np.random.default_rng(30 + pt)
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
            ref = orc.orth_backward(g, ys[nf - 1].cpu().numpy().astype(np.float64), s)
            assert orc.rel_l2(outs[1][nf - 1], ref) < TOL


@pytest.mark.parametrize("pt", [2, 3])
def test_orth_system_matrix_forward(cuda, pt):
    """Types 2 / 3 (non-TOF) forward projections through the ray-major copy
    of the tube weights (tuning siddon_bp_matrix = 1, same type both ways)
    against the tracer and the FP64 oracle, frames batched and single."""
    import ctypes

    import torch
    from omega_b200 import _native
    o = _opts("pet_mini", pt)
    o.initProj()
    g = orc.Geometry(o)
    n = int(o.N[0])
    rng = np.random.default_rng(40 + pt)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for s in range(g.n_subsets):
        m = o.measurementCount(s)
        for nf in (1, 3):
            xs = _t(rng.uniform(0.5, 2.0, (nf, n)), cuda)
            outs = []
            for mat in (0, 1, 1):
                o.tuning = {"siddon_bp_matrix": mat}
                y = torch.empty((nf, m), device=cuda)
                _native.call("omb_forward_frames", o._handle, s, nf, ctypes.c_void_p(xs.data_ptr()), n,
                             ctypes.c_void_p(y.data_ptr()), m, st)
                outs.append(y.cpu().numpy())
            assert np.array_equal(outs[1].view(np.uint32), outs[2].view(np.uint32))
            for f in range(nf):
                assert orc.rel_l2(outs[1][f], outs[0][f]) < 1e-6, (s, nf, f)
            ref = orc.orth_forward(g, xs[nf - 1].cpu().numpy().astype(np.float64), s)
            assert orc.rel_l2(outs[1][nf - 1], ref) < TOL
