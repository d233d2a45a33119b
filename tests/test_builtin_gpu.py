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
                   prior_grad=lambda x: io.rdp_gradient(x, shape, 2.0, 0.002, g.epps))
    plain = orc.osem(g, ys, np.ones(g.n_img), 2)
    x = out.ravel(order='F')
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)
    assert orc.rel_l2(ref, plain) > 1e-3  # the prior changes the result
