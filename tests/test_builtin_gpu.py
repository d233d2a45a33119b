"""The built-in reconstruction entry (reconstructions_main /
reconstructions_mainCT, native loop omb_reconstruct) against the custom-loop
classes and the FP64 oracle: OSEM on PET sinograms (with corrections and
randoms, TOF), PDHG+TV on cone-beam CT, eager and CUDA-graph replays."""
import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _pet_data(o, seed):
    g = orc.Geometry(o)
    rng = np.random.default_rng(seed)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    # full measurement vector in the reference's order (before subset reordering)
    full = make_options(o._cfg_name)
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    gf = orc.Geometry(full)
    y = rng.poisson(orc.forward(gf, truth, 0) * 200).astype(np.float32) / 200
    return g, y


@pytest.mark.parametrize("name,graph", [("pet_mini", True), ("pet_mini", False), ("pet_mini_tof", True),
                                        ("pet_stype1", True)])
def test_builtin_osem_matches_oracle(cuda, name, graph):
    from omega_b200 import reconstruction as rec
    o = make_options(name)
    o._cfg_name = name
    g, y = _pet_data(o, 1)
    o.SinM = y.copy()
    o.OSEM = True
    o.Niter = 2
    o.use_graph = graph
    out, fp = rec.reconstructions_main(o)
    assert out.shape == (g.nx, g.ny, g.nz, 1) and fp.size == 0
    x = out.ravel(order='F')
    # the oracle on the same subset-ordered measurements
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    ref = orc.osem(g, ys, np.ones(g.n_img), 2)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)


def test_builtin_osem_equals_custom_loop(cuda):
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    o._cfg_name = "pet_mini"
    g, y = _pet_data(o, 2)
    o.SinM = y.copy()
    o.OSEM = True
    o.Niter = 3
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    x = rec.OSEM(o, m).iterate(3).cpu().numpy()
    # float atomics: equal up to the order of the backprojection's additions
    assert orc.rel_l2(out.ravel(order='F'), x) < 1e-6


def test_builtin_pdhg_ct_matches_custom_loop_and_oracle(cuda):
    from omega_b200 import reconstruction as rec
    o = make_options("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(3)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    counts = 1e4 * np.exp(-orc.bdd_forward(g, truth, -1))
    o.SinM = rng.poisson(counts).astype(np.float32) + 1
    o.PDHG = True
    o.TV = True
    o.beta = 0.05
    o.Niter = 5
    o.x0 = np.zeros(g.n_img, dtype=np.float32)
    out, _ = rec.reconstructions_mainCT(o)
    tau = o.tau_used
    assert tau > 0
    y = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')   # linearised by the entry
    custom = rec.PDHG(o, y, beta=0.05, tau=tau, x0=np.zeros(g.n_img)).iterate(5).cpu().numpy()
    assert orc.rel_l2(out.ravel(order='F'), custom) < 1e-6
    ref = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau, 0.05, 1e-4)
    assert orc.rel_l2(out.ravel(order='F'), ref) < 1e-4, orc.rel_l2(out.ravel(order='F'), ref)
    # the power-method step agrees with the custom loop's estimate
    assert abs(tau * rec.power_method(o) - 1.0) < 1e-2


@pytest.mark.parametrize("tvtype", [4, 6])
def test_builtin_pdhg_ct_tv_variants(cuda, tvtype):
    """PDHG with SATV (TVtype 4) and the weighted TV (TVtype 6): the variant
    gradient is added to A^T p before the primal step."""
    from omega_b200 import reconstruction as rec
    from oracle import image_oracle as io
    o = make_options("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(4)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    counts = 1e4 * np.exp(-orc.bdd_forward(g, truth, -1))
    o.SinM = rng.poisson(counts).astype(np.float32) + 1
    o.PDHG = True
    o.TV = True
    o.TVtype = tvtype
    o.SATVPhi = 0.01
    o.beta = 5.0     # strong enough that the TV form shows in 5 iterations
    o.Niter = 5
    o.x0 = np.zeros(g.n_img, dtype=np.float32)
    out, _ = rec.reconstructions_mainCT(o)
    tau = o.tau_used
    y = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    name = "satv" if tvtype == 4 else "tvw1"
    shape = (g.nx, g.ny, g.nz)
    ref = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau, 5.0, 1e-4,
                      tv_grad=lambda v: io.tv_gradient_variant(v, shape, name, 1e-4, 5.0, sigma=0.01))
    assert orc.rel_l2(out.ravel(order='F'), ref) < 1e-4, orc.rel_l2(out.ravel(order='F'), ref)
    plain = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau, 5.0, 1e-4)
    assert orc.rel_l2(plain, ref) > 1e-3   # the variant changes the result


@pytest.mark.parametrize("l2,diff_type", [(True, 0), (False, 0), (True, 1)])
def test_proxtv_kernels_match_oracle(cuda, l2, diff_type):
    """omb_proxtv_dual and omb_proxtv_divergence against the restatement
    (pinned to the reference's ProxTV kernels), the ball active on part of
    the image."""
    import ctypes

    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    from oracle import image_oracle as io
    shape = (21, 17, 9)
    n = int(np.prod(shape))
    rng = np.random.default_rng(54)
    x = rng.uniform(0.0, 1.0, n).astype(np.float32)
    q = rng.normal(0.0, 0.3, (3, n)).astype(np.float32)
    rhs = rng.normal(0.0, 1.0, n).astype(np.float32)
    X, Q, R = (torch.tensor(a, device=cuda) for a in (x, q, rhs))
    st = _stream(cuda)
    _native.call("omb_proxtv_dual", ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(Q.data_ptr()), *shape, 0.7, 0.25,
                 1 if l2 else 0, diff_type, st)
    _native.call("omb_proxtv_divergence", ctypes.c_void_p(Q.data_ptr()), ctypes.c_void_p(R.data_ptr()), *shape,
                 diff_type, st)
    want_q = io.proxtv_dual(x.astype(np.float64), q.astype(np.float64), shape, 0.7, 0.25, l2, diff_type)
    want_r = rhs - io.proxtv_divergence(want_q, shape, diff_type)
    assert orc.rel_l2(Q.cpu().numpy().ravel(), want_q.ravel()) < 1e-6
    assert orc.rel_l2(R.cpu().numpy(), want_r) < 1e-6


def test_builtin_pdhg_ct_proxtv(cuda):
    """PDHG with the proximal TV (options.ProxTV) through the built-in entry
    against the FP64 loop."""
    from omega_b200 import reconstruction as rec
    o = make_options("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(5)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    counts = 1e4 * np.exp(-orc.bdd_forward(g, truth, -1))
    o.SinM = rng.poisson(counts).astype(np.float32) + 1
    o.PDHG = True
    o.ProxTV = True
    # beta and the TV dual step large enough that the ball projection acts
    # and the TV term moves the image by ~15 % in 5 iterations
    o.beta = 5.0
    o.sigma2CP = 1000.0
    o.Niter = 5
    o.x0 = np.zeros(g.n_img, dtype=np.float32)
    out, _ = rec.reconstructions_mainCT(o)
    tau = o.tau_used
    y = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ref = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau, 5.0, 1e-4,
                      prox=dict(sigma2=1000.0, l2=True, diff_type=0))
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 1e-4, orc.rel_l2(x, ref)
    plain = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau, 0.0, 1e-4)
    assert orc.rel_l2(plain, ref) > 1e-2


@pytest.mark.parametrize("l2,three_d", [(True, True), (False, True), (True, False), (False, False)])
def test_proxtgv_kernel_matches_oracle(cuda, l2, three_d):
    """omb_proxtgv_step against the restatement (pinned to the reference's
    six TGV kernels), both balls active on part of the image."""
    import ctypes

    import torch
    from omega_b200 import _native
    from omega_b200.reconstruction import _stream
    from oracle import image_oracle as io
    shape = (37, 19, 11)
    n = int(np.prod(shape))
    nr, nv = (6, 3) if three_d else (3, 2)
    rng = np.random.default_rng(63)
    x = rng.uniform(0.0, 1.0, n).astype(np.float32)
    q = rng.normal(0.0, 0.3, (3, n)).astype(np.float32)
    r = rng.normal(0.0, 0.2, (nr, n)).astype(np.float32)
    v = rng.normal(0.0, 0.2, (nv, n)).astype(np.float32)
    rhs = rng.normal(0.0, 1.0, n).astype(np.float32)
    X, Q, R, V, H = (torch.tensor(a, device=cuda) for a in (x, q, r, v, rhs))
    _native.call("omb_proxtgv_step", *(ctypes.c_void_p(t.data_ptr()) for t in (X, Q, R, V, H)), *shape, 0.7, 0.3,
                 0.2, 0.9, 0.05, 1 if l2 else 0, 1 if three_d else 0, _stream(cuda))
    want = io.proxtgv_step(*(a.astype(np.float64) for a in (x, q, r, v, rhs)), shape, 0.7, 0.3, 0.2, 0.9, 0.05,
                           l2=l2, three_d=three_d)
    for got, w in zip((Q, R, V, H), want):
        assert orc.rel_l2(got.cpu().numpy().ravel(), w.ravel()) < 1e-6, orc.rel_l2(got.cpu().numpy().ravel(),
                                                                                    w.ravel())


@pytest.mark.parametrize("use2d,K", [(False, None), (True, None), (False, 2)])
def test_builtin_pdhg_ct_tgv(cuda, use2d, K):
    """PDHG with TGV (options.TGV; 3-D or use2DTGV) through the built-in
    entry against the FP64 loop; with K, also the filtering-based
    measurement preconditioner, whose inverse filter takes sigma beta."""
    from omega_b200 import filters
    from omega_b200 import reconstruction as rec
    o = make_options("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(7)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    counts = 1e4 * np.exp(-orc.bdd_forward(g, truth, -1))
    o.SinM = rng.poisson(counts).astype(np.float32) + 1
    o.PDHG = True
    o.TGV = True
    o.use2DTGV = use2d
    # balls and the dual step large enough that TGV moves the image by ~13 %
    o.alpha0TGV = 5.0
    o.alpha1TGV = 10.0
    o.sigma2CP = 1000.0
    beta = 1.0 if K is None else 2.0
    o.beta = beta
    o.Niter = 5
    o.x0 = np.zeros(g.n_img, dtype=np.float32)
    mf = None
    if K is not None:
        o.precondTypeMeas = np.array([False, True])
        o.filteringIterations = K
        o.filterWindow = "hann"
        o.tauCP = 2e-5
    out, _ = rec.reconstructions_mainCT(o)
    tau = o.tau_used
    y = np.asarray(o.SinM, dtype=np.float32).ravel(order='F').astype(np.float64)
    if K is not None:
        nr = int(o.nRowsD)
        nf, f0, ff, _, _ = filters.pdhg_row_filters(nr, beta, "hann")
        mf = dict(filter0=f0, ffilter=ff, nf=nf, rows=nr, K=K, tau2=float(np.float32(2e-5)))
    tg = dict(alpha0=5.0, alpha1=10.0, sigma2=1000.0, l2=True, three_d=not use2d)
    ref = orc.pdhg_tv(g, y, np.zeros(g.n_img), 5, tau, beta, 1e-4, tgv=tg, meas_filter=mf)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 1e-4, orc.rel_l2(x, ref)
    plain = orc.pdhg_tv(g, y, np.zeros(g.n_img), 5, tau, 0.0, 1e-4, meas_filter=mf)
    assert orc.rel_l2(plain, ref) > 1e-2


@pytest.mark.parametrize("rows,window", [(100, "hann"), (512, "hamming"), (37, "parzen")])
def test_row_filter_kernel(cuda, rows, window):
    """omb_row_filter (circular convolution with the taps) against the
    reference's Fourier-domain filtering restated in FP64."""
    import ctypes

    import torch
    from omega_b200 import _native, filters
    from omega_b200.reconstruction import _stream
    nf, f0, ff, h, hinv = filters.pdhg_row_filters(rows, 1.0, window)
    rng = np.random.default_rng(rows)
    v = rng.normal(size=rows * 203).astype(np.float32)
    V, H, HI = (torch.tensor(a, device=cuda) for a in (v, h, hinv))
    out = torch.empty_like(V)
    for taps, filt, inv in ((H, f0, False), (HI, ff, True)):
        _native.call("omb_row_filter", ctypes.c_void_p(V.data_ptr()), ctypes.c_void_p(out.data_ptr()), rows, 203,
                     ctypes.c_void_p(taps.data_ptr()), nf, _stream(cuda))
        want = orc.row_filter_fft(v, rows, nf, filt, inverse=inv)
        assert orc.rel_l2(out.cpu().numpy(), want) < 1e-6, orc.rel_l2(out.cpu().numpy(), want)


@pytest.mark.parametrize("K", [2, 0])
def test_builtin_pdhg_ct_measurement_filter(cuda, K):
    """PDHG + TV with the filtering-based measurement preconditioner
    (precondTypeMeas[1]): K filtering iterations with the inverse-filtered
    dual step, then the plain steps with tauCP; K = 0 filters every
    residual."""
    from omega_b200 import filters
    from omega_b200 import reconstruction as rec
    o = make_options("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(6)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    counts = 1e4 * np.exp(-orc.bdd_forward(g, truth, -1))
    o.SinM = rng.poisson(counts).astype(np.float32) + 1
    o.PDHG = True
    o.TV = True
    o.beta = 0.05
    o.Niter = 5
    o.x0 = np.zeros(g.n_img, dtype=np.float32)
    o.precondTypeMeas = np.array([False, True])
    o.filteringIterations = K
    o.filterWindow = "hann"
    # the step after the filtering iterations: 1 / the FP64 power-method eigenvalue of A^T A
    xv = np.abs(rng.normal(size=g.n_img))
    xv /= np.linalg.norm(xv)
    for _ in range(20):
        bv = orc.bdd_backward(g, orc.bdd_forward(g, xv, -1), -1)
        L = float(bv @ xv / (xv @ xv))
        xv = bv / np.linalg.norm(bv)
    tau2 = float(np.float32(1.0 / L))
    o.tauCP = tau2
    out, _ = rec.reconstructions_mainCT(o)
    tau_f = o.tau_used
    assert tau_f > 0
    y = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    nr = int(o.nRowsD)
    nf, f0, ff, _, _ = filters.pdhg_row_filters(nr, 1.0, "hann")
    mf = dict(filter0=f0, ffilter=ff, nf=nf, rows=nr, K=K, tau2=tau2)
    ref = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau_f, 0.05, 1e-4, meas_filter=mf)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 1e-4, orc.rel_l2(x, ref)
    plain = orc.pdhg_tv(g, y.astype(np.float64), np.zeros(g.n_img), 5, tau_f, 0.05, 1e-4)
    assert orc.rel_l2(plain, ref) > 1e-3


@pytest.mark.parametrize("shape,window", [((32, 32, 5), "hann"), ((45, 37, 3), "hamming"), ((128, 100, 2), "cosine")])
def test_image_filter_kernel(cuda, shape, window):
    """omb_image_filter (separable circular convolution of the x and y
    lines) against filtering2D restated with 2-D FFTs in FP64."""
    import ctypes

    import torch
    from omega_b200 import _native, filters
    from omega_b200.reconstruction import _stream
    nf, F, h = filters.image_filter_2d(shape[0], window)
    n = int(np.prod(shape))
    rng = np.random.default_rng(8)
    v = rng.normal(size=n).astype(np.float32)
    G = torch.tensor(v, device=cuda)
    T = torch.empty_like(G)
    H = torch.tensor(h, device=cuda)
    _native.call("omb_image_filter", ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(T.data_ptr()), *shape,
                 ctypes.c_void_p(H.data_ptr()), nf, _stream(cuda))
    want = orc.image_filter_fft(v.astype(np.float64), shape, nf, F)
    assert orc.rel_l2(G.cpu().numpy(), want) < 1e-6, orc.rel_l2(G.cpu().numpy(), want)


@pytest.mark.parametrize("K", [2, 0, 9])
def test_builtin_pdhg_ct_image_filter(cuda, K):
    """PDHG + TV with the filtering-based image preconditioner
    (precondTypeImage[5]): A^T p plus the TV term filtered in iterations
    k < K, then the unfiltered power-method step; K = 0 filters the first
    iteration only."""
    from omega_b200 import filters
    from omega_b200 import reconstruction as rec
    o = make_options("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(9)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    counts = 1e4 * np.exp(-orc.bdd_forward(g, truth, -1))
    o.SinM = rng.poisson(counts).astype(np.float32) + 1
    o.PDHG = True
    o.TV = True
    o.beta = 0.05
    o.Niter = 5
    o.x0 = np.zeros(g.n_img, dtype=np.float32)
    o.precondTypeImage = np.array([0, 0, 0, 0, 0, 1, 0], bool)
    o.filteringIterations = K
    o.filterWindow = "hann"
    out, _ = rec.reconstructions_mainCT(o)
    tau_f, tau2 = o.tau_used, o.tau_used2
    assert tau_f > 0 and (tau2 > 0) == (0 < K < 5)
    y = np.asarray(o.SinM, dtype=np.float32).ravel(order='F').astype(np.float64)
    nf, F, _ = filters.image_filter_2d(g.nx, "hann")
    imf = dict(nf=nf, F=F, K=K, tau2=tau2)
    ref = orc.pdhg_tv(g, y, np.zeros(g.n_img), 5, tau_f, 0.05, 1e-4, img_filter=imf)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 1e-4, orc.rel_l2(x, ref)
    plain = orc.pdhg_tv(g, y, np.zeros(g.n_img), 5, tau_f, 0.05, 1e-4)
    assert orc.rel_l2(plain, ref) > 1e-3


def test_builtin_osl_osem_rdp_matches_oracle(cuda):
    from omega_b200 import reconstruction as rec
    from oracle import image_oracle as io
    o = make_options("pet_mini")
    o._cfg_name = "pet_mini"
    g, y = _pet_data(o, 4)
    o.SinM = y.copy()
    o.OSL_OSEM = True
    o.RDP = True
    o.RDP_gamma = 2.0
    # one-step-late is stable only for small weights: at beta = 0.02 this
    # case is chaotic (a 1e-6 change of x0 moves the result by 30 %)
    o.beta = 0.002
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    ref = orc.osem(g, ys, np.ones(g.n_img), 2,
                   prior_grad=lambda x: io.rdp_gradient(x, shape, 2.0, 0.002, g.epps, clamp=True))
    plain = orc.osem(g, ys, np.ones(g.n_img), 2)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, plain) > 1e-3  # the prior changes the result
