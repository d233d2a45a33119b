"""The L-filter and FMH priors (priors.h:54-97) with the MATLAB prepass's
weights (lfilter_weights.m, fmhWeights.m): the weights against hand-worked
values, the restatements against the pinned median root prior and an
explicit per-voxel statement, the CUDA gradients against the restatements,
and OSL-OSEM with each prior against the oracle loop."""
import ctypes
import types

import numpy as np
import pytest

from oracle import image_oracle as io
from oracle import oracle as orc

SHAPE = (12, 11, 9)


def _opts(shape=SHAPE, **kw):
    o = types.SimpleNamespace(Nx=shape[0], Ny=shape[1], Nz=shape[2], FOVa_x=float(shape[0]),
                              FOVa_y=float(shape[1]), axial_fov=float(shape[2]), Ndx=1, Ndy=1, Ndz=1,
                              a_L=np.empty(0), fmh_weights=np.empty(0), oneD_weights=False, fmh_center_weight=4.)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _image(seed, shape=SHAPE):
    rng = np.random.default_rng(seed)
    return np.round(rng.uniform(0.5, 1.5, int(np.prod(shape))), 2)   # rounded: ties in most windows


def test_lfilter_weights_follow_the_prepass():
    from omega_b200 import priors
    # 2-D, unit voxels: 0.5 exp(x sqrt 2), x = -1.5, -0.75, 0: centre / 1, axes / 1, diagonals / sqrt 2
    a1 = 0.5 * np.exp(np.array([-1.5, -0.75, 0.0]) * np.sqrt(2.0))
    d, ax, c = a1[0] / np.sqrt(2.0), a1[1], a1[2]
    want = np.array([d, ax, d, ax, c, ax, d, ax, d])
    assert np.allclose(priors.lfilter_weights(_opts(Ndz=0)), want / want.sum(), rtol=1e-6)
    w3 = priors.lfilter_weights(_opts())
    assert w3.size == 27 and abs(float(w3.sum()) - 1) < 1e-6 and np.array_equal(w3, w3[::-1])
    # the 3-D space diagonal uses sqrt(sqrt(dx^2 + dy^2) + dz^2), as lfilter_weights.m writes it
    assert np.isclose(w3[0] / w3[13], a1[0] / np.sqrt(np.sqrt(2.0) + 1.0) / a1[2], rtol=1e-6)
    # one-dimensional: the tabulated 9-value set mirrored, unnormalised
    t = [-0.01899, 0.02904, 0.06965, 0.23795, 0.36469]
    assert np.array_equal(priors.lfilter_weights(_opts(Ndz=0, oneD_weights=True)),
                          np.asarray(t + t[:-1][::-1], np.float32))
    # 125 values: the Laplace curve on linspace(-4, 0, 63), mirrored, normalised
    h = 0.5 * np.exp(np.linspace(-4.0, 0.0, 63) * np.sqrt(2.0))
    h = np.concatenate([h, h[:-1][::-1]])
    assert np.allclose(priors.lfilter_weights(_opts(Ndx=2, Ndy=2, Ndz=2, oneD_weights=True)), h / h.sum(),
                       rtol=1e-6)
    with pytest.raises(ValueError, match="numerical integration"):
        priors.lfilter_weights(_opts(oneD_weights=True))
    user = np.linspace(0, 1, 27).astype(np.float32)
    assert np.array_equal(priors.lfilter_weights(_opts(a_L=user)), user)
    with pytest.raises(ValueError, match="a_L"):
        priors.lfilter_weights(_opts(a_L=user[:9]))


def test_fmh_weights_follow_the_prepass():
    from omega_b200 import priors
    r2 = np.sqrt(2.0)
    # 2-D, unit voxels, centre weight 4: kerroin = 4^(1/4) = sqrt 2; the diagonals [1, 4, 1],
    # the axes [sqrt 2, 4, sqrt 2], each normalised; columns diagonal, x, diagonal, y
    W = priors.fmh_weights(_opts(Ndz=0)).reshape((3, 4), order='F')
    diag = np.array([1.0, 4.0, 1.0]) / 6.0
    axis = np.array([r2, 4.0, r2]) / (4.0 + 2 * r2)
    assert np.allclose(W, np.stack([diag, axis, diag, axis], axis=1), rtol=1e-6)
    W3 = priors.fmh_weights(_opts()).reshape((3, 13), order='F')
    assert np.allclose(W3.sum(axis=0), 1.0, rtol=1e-6)
    # the space diagonals (columns 1, 3, 7, 9) over sqrt(3) |i|, the z axis (5) over |i|
    sd = np.array([r2 / np.sqrt(3.0), 4.0, r2 / np.sqrt(3.0)])
    assert np.allclose(W3[:, 0], sd / sd.sum(), rtol=1e-6)
    assert np.allclose(W3[:, 4], axis, rtol=1e-6)
    assert np.allclose(W3[:, 9:], W, rtol=1e-6)
    # a single slice takes the 2-D set even with Ndz = 1
    assert priors.fmh_weights(_opts(shape=(12, 11, 1))).size == 12
    with pytest.raises(ValueError, match="Ndx = Ndy = Ndz"):
        priors.fmh_weights(_opts(Ndx=2, Ndy=2, Ndz=1))


@pytest.mark.parametrize("m", [(1, 1, 1), (2, 2, 2), (1, 1, 0)])
def test_lfilter_with_the_median_weight_is_the_median_root_prior(m):
    """a_L one at the middle rank makes the L-filter the median root prior,
    whose median is pinned to the reference's medianFilter3D."""
    u = _image(sum(m))
    n = (2 * m[0] + 1) ** (3 if m[2] else 2)
    a = np.zeros(n)
    a[n // 2] = 1.0
    for no_norm in (False, True):
        assert np.array_equal(io.lfilter_gradient(u, SHAPE, m, a, 0.3, 1e-8, no_norm),
                              io.mrp_gradient(u, SHAPE, m, 0.3, 1e-8, no_norm))


def _mir(i, n):
    return -i - 1 if i < 0 else (2 * n - 1 - i if i >= n else i)


@pytest.mark.parametrize("shape", [(7, 6, 5), (7, 6, 1)])
def test_fmh_restatement_against_explicit_lines(shape):
    """The offsets-grid columns priors.h selects resolve, for Ndx = 1, to the
    lines through the voxel listed here by hand: 13 in 3-D, and with one
    slice 4 (the first four 3-D lines, whose z steps mirror onto the slice)."""
    rng = np.random.default_rng(4)
    u = _image(5, shape)
    W = rng.uniform(0.1, 1.0, (3, 13))
    nx, ny, nz = shape
    U = u.reshape((nz, ny, nx))
    # line ii runs from column ii through the centre (13) to column 26 - ii; column a is the offset
    # (a % 3 - 1, a // 3 % 3 - 1, a // 9 - 1), so the line's step is minus that of column ii
    steps = [(1 - a % 3, 1 - (a // 3) % 3, 1 - a // 9) for a in range(13)]
    lines = 4 if nz == 1 else 13
    Wl = W[:, :lines]
    want = np.zeros(u.size)
    n = 0
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                vals = []
                for ii in range(lines):
                    si, sj, sk = steps[ii]
                    acc = 0.0
                    for e, t in enumerate((-1, 0, 1)):
                        acc += Wl[e, ii] * U[_mir(z + t * sk, nz), _mir(y + t * sj, ny), _mir(x + t * si, nx)]
                    vals.append(acc)
                vals.append(U[z, y, x])
                med = np.median(vals)
                want[n] = 0.7 * (U[z, y, x] - med) / (med + 1e-8)
                n += 1
    got = io.fmh_gradient(u, shape, (1, 1, 1), Wl.ravel(order='F'), 0.7, 1e-8)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-14)


def test_median_filter_priors_validate():
    from omega_b200 import _native
    L = _native.lib()
    p = ctypes.c_void_p(16)
    f = ctypes.c_float
    for name in ("omb_lfilter_gradient", "omb_fmh_gradient"):
        fn = getattr(L, name)
        # NULL weights, a (2, 2, 1) window, a window wider than the image: refused before any launch
        assert fn(p, p, 8, 8, 8, 1, 1, 1, None, f(1e-8), f(1.0), 0, None) != 0
        assert fn(p, p, 8, 8, 8, 2, 2, 1, p, f(1e-8), f(1.0), 0, None) != 0
        assert fn(p, p, 8, 8, 1, 2, 2, 2, p, f(1e-8), f(1.0), 0, None) != 0
    assert L.omb_lfilter_gradient(p, p, 8, 8, 8, 3, 3, 3, p, f(1e-8), f(1.0), 0, None) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("m,shape,no_norm", [((1, 1, 1), SHAPE, False), ((2, 2, 2), SHAPE, True),
                                             ((1, 1, 0), SHAPE, False), ((1, 1, 1), (12, 11, 1), True)])
@pytest.mark.parametrize("kind", ["L", "FMH"])
def test_kernels_match_restatements(cuda, kind, m, shape, no_norm):
    import torch
    from omega_b200 import _native, priors
    from omega_b200.reconstruction import _stream
    u = _image(9, shape).astype(np.float32)
    o = _opts(shape=shape, Ndx=m[0], Ndy=m[1], Ndz=m[2])
    w = priors.lfilter_weights(o) if kind == "L" else priors.fmh_weights(o)
    U = torch.tensor(u, device=cuda)
    Wd = torch.tensor(w, device=cuda)
    out = torch.full((u.size,), 0.5, device=cuda)
    _native.call("omb_lfilter_gradient" if kind == "L" else "omb_fmh_gradient", ctypes.c_void_p(U.data_ptr()),
                 ctypes.c_void_p(out.data_ptr()), *shape, *m, ctypes.c_void_p(Wd.data_ptr()), 1e-8, 0.3,
                 1 if no_norm else 0, _stream(cuda))
    ref = io.lfilter_gradient if kind == "L" else io.fmh_gradient
    want = 0.5 + ref(u.astype(np.float64), shape, m, w.astype(np.float64), 0.3, 1e-8, no_norm)
    assert np.max(np.abs(out.cpu().numpy() - want)) < 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["L", "FMH"])
def test_builtin_bsrem_with_median_filter_priors(cuda, kind):
    """BSREM with each prior against the oracle loop.  BSREM's MAP step keeps
    the image >= epps; one-step-late OSEM on this phantom drives voxels the
    rays barely reach negative through sens + dU < 0, where FP32 and FP64
    part ways, so the built-in check uses BSREM, as the weighted mean's does."""
    from conftest import make_options
    from omega_b200 import priors
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(12)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), rng.uniform(0.5, 2.0, g.n_img), 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.BSREM = True
    setattr(o, kind, True)
    o.beta = 0.5
    o.Niter = 2
    lam = np.array([0.2, 0.12], np.float32)
    o.lambdaN = lam
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    nd = (int(o.Ndx), int(o.Ndy), int(o.Ndz))
    w = (priors.lfilter_weights(o) if kind == "L" else priors.fmh_weights(o)).astype(np.float64)
    f = io.lfilter_gradient if kind == "L" else io.fmh_gradient
    ref = orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam,
                      prior_grad=lambda v: f(v, shape, nd, w, 0.5, g.epps))
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, orc.relaxed(g, ys, np.ones(g.n_img), 2, "BSREM", lam=lam,
                                      prior_grad=lambda v: 0.0 * v)) > 1e-3
