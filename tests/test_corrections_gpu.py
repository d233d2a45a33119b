"""PET corrections in the type-1 projector kernels (normalisation x scatter x
LOR attenuation as one weight per measurement, attenuation image line
integrals): CUDA against the FP64 oracle (pinned to the reference CPU
projector by test_corrections_oracle.py) at 1e-5 relative L2, through the
projectorClass attributes of the reference (normalization, vaimennus,
CTAttenuation, corrVector) and through the frame-batched and fixed-point
entry points."""
import ctypes

import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _corrected(name, seed, image_atten=True, **extra):
    o = make_options(name)
    for k, v in extra.items():
        setattr(o, k, v)
    rng = np.random.default_rng(seed)
    total = int(np.ravel(o.nTotMeas)[-1])
    n_img = int(np.ravel(o.N)[0])
    o.normalization_correction = 1
    o.normalization = rng.uniform(0.5, 1.5, total).astype(np.float32)
    o.attenuation_correction = 1
    o.CTAttenuation = image_atten
    o.vaimennus = (0.0096 * rng.uniform(0.5, 1.5, n_img) if image_atten else
                   rng.uniform(0.3, 1.0, total)).astype(np.float32)
    o.additionalCorrection = 1
    o.corrVector = rng.uniform(0.8, 1.2, total).astype(np.float32)
    o.initProj()
    g = orc.Geometry(o)
    # after initProj the vectors are in subset order, as the kernels read them
    w = o.normalization.astype(np.float64) * o.corrVector
    if not image_atten:
        w = w * o.vaimennus
    g.w = w
    g.mu = o.vaimennus.astype(np.float64) if image_atten else None
    return o, g, rng


@pytest.mark.parametrize("name,image_atten", [("pet_mini", True), ("pet_mini", False), ("pet_mini_tof", True),
                                              ("pet_stype1", True), ("pet_odd_span1", True)])
def test_corrected_projections_match_oracle(cuda, name, image_atten):
    o, g, rng = _corrected(name, 7, image_atten)
    x = rng.uniform(0.5, 2.0, g.n_img)
    for s in range(g.n_subsets):
        fp = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        assert orc.rel_l2(fp, orc.forward(g, x, s)) < TOL, s
        y = rng.uniform(0.0, 2.0, g.rays(s) * g.nbins)
        bp, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref_bp, ref_s = orc.backward(g, y, s, sens=True)
        assert orc.rel_l2(bp.cpu().numpy(), ref_bp) < TOL, s
        assert orc.rel_l2(sens.cpu().numpy(), ref_s) < TOL, s


def test_corrected_frames_and_fixed_point(cuda):
    """Frame batches (both frame layouts) and the int64 backprojection carry
    the same corrections."""
    import torch
    from omega_b200 import _native
    o, g, rng = _corrected("pet_mini", 8, use_64bit_atomics=True)
    n, m = g.n_img, o.measurementCount(-1)
    frames = 5
    imgs = rng.uniform(0.5, 2.0, (frames, n))
    ys = rng.uniform(0.0, 2.0, (frames, m))
    cut = np.cumsum([0] + [g.rays(s) for s in range(g.n_subsets)])
    ref_fp = [np.concatenate([orc.forward(g, imgs[f], s) for s in range(g.n_subsets)]) for f in range(frames)]
    ref_bp = [sum(orc.backward(g, ys[f, cut[s]:cut[s + 1]], s) for s in range(g.n_subsets)) for f in range(frames)]
    X, Yin = _t(imgs, cuda), _t(ys, cuda)
    Y = torch.empty((frames, m), device=cuda)
    B = torch.empty((frames, n), device=cuda)
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    for lay in (0, 1):
        o.tuning = {"siddon_frame_layout": lay, "siddon_frames_per_walk": 8}
        _native.call("omb_forward_frames", o._handle, -1, frames, ctypes.c_void_p(X.data_ptr()), n,
                     ctypes.c_void_p(Y.data_ptr()), m, st)
        _native.call("omb_backward_frames", o._handle, -1, frames, ctypes.c_void_p(Yin.data_ptr()), m,
                     ctypes.c_void_p(B.data_ptr()), n, st)
        y, b = Y.cpu().numpy(), B.cpu().numpy()
        for f in range(frames):
            assert orc.rel_l2(y[f], ref_fp[f]) < TOL, (lay, f)
            assert orc.rel_l2(b[f], ref_bp[f]) < TOL, (lay, f)
    y0 = rng.uniform(0.0, 2.0, g.rays(0))
    a = o.backwardProject(_t(y0, cuda), 0).cpu().numpy()
    bb = o.backwardProject(_t(y0, cuda), 0).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), bb.view(np.uint32))
    assert orc.rel_l2(a, orc.backward(g, y0, 0)) < TOL


def test_corrections_rejected_where_not_built(cuda):
    from omega_b200 import _native
    # projector type 4 with corrections
    with pytest.raises(_native.NativeError):
        o, g, rng = _corrected("pet_mini4", 9)
        o.forwardProject(_t(np.ones(g.n_img), cuda), 0)
    # wrong vector length
    o = make_options("pet_mini")
    o.normalization_correction = 1
    o.normalization = np.ones(5, dtype=np.float32)
    with pytest.raises(ValueError):
        o.initProj()


@pytest.mark.parametrize("name", ["pet_mini", "pet_mini_tof"])
def test_osem_with_corrections_and_randoms_matches_oracle(cuda, name):
    """Ordinary-Poisson OSEM: corrected projector pair, sensitivity with the
    same corrections, randoms added before the ratio."""
    from omega_b200 import reconstruction as rec
    o = make_options(name)
    rng = np.random.default_rng(11)
    total = int(np.ravel(o.nTotMeas)[-1])
    n_img = int(np.ravel(o.N)[0])
    o.normalization_correction = 1
    o.normalization = rng.uniform(0.7, 1.3, total).astype(np.float32)
    o.attenuation_correction = 1
    o.vaimennus = (0.0096 * rng.uniform(0.5, 1.5, n_img)).astype(np.float32)
    o.randoms_correction = 1
    o.SinDelayed = rng.uniform(0.05, 0.2, total).astype(np.float32)
    o.initProj()
    g = orc.Geometry(o)
    g.w = o.normalization.astype(np.float64)
    g.mu = o.vaimennus.astype(np.float64)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    cut = np.cumsum([0] + [g.rays(s) for s in range(g.n_subsets)])
    rnd = [o.SinDelayed[cut[s]:cut[s + 1]].astype(np.float64) for s in range(g.n_subsets)]
    ys = [rng.poisson(orc.forward(g, truth, s) * 1000 + np.tile(rnd[s], g.nbins) * 1000).astype(np.float32) / 1000
          for s in range(g.n_subsets)]
    # the flat measurement vector: TOF bins outermost, subsets inside
    n = np.diff(cut)
    m = np.concatenate([np.concatenate([ys[s][b * n[s]:(b + 1) * n[s]] for s in range(g.n_subsets)])
                        for b in range(g.nbins)])
    x = rec.OSEM(o, m).iterate(2).cpu().numpy()
    ref = orc.osem(g, ys, np.ones(g.n_img), 2, randoms=rnd)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
