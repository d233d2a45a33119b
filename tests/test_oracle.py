"""Pins the FP64 oracle (oracle/siddon_oracle.c) to the reference's own CPU
projector outputs stored in the golden fixtures, and checks its adjointness
and the restated OSEM loop.  CPU only."""
import numpy as np
import pytest

from conftest import load_golden, make_options
from oracle import oracle as orc

# fixtures hold the reference's FP64 results rounded to float32
TOL = 1e-6


@pytest.mark.parametrize("name", ["pet_mini", "pet_tof_small"])
def test_oracle_forward_matches_reference(name):
    o = make_options(name)
    g = orc.Geometry(o)
    p = load_golden("proj", name)
    keys = [k for k in p if k.startswith("fp_")]
    assert keys
    for k in keys:
        y = orc.forward(g, p["image"], int(k[3:]))
        assert orc.rel_l2(y, p[k]) < TOL, k


@pytest.mark.parametrize("name", ["pet_mini", "pet_tof_small"])
def test_oracle_backward_matches_reference(name):
    o = make_options(name)
    g = orc.Geometry(o)
    p = load_golden("proj", name)
    bp, sens = orc.backward(g, p["bp_in_0"], 0, sens=True)
    assert orc.rel_l2(bp, p["bp_0"]) < TOL
    assert orc.rel_l2(sens, p["sens_0"]) < TOL


@pytest.mark.parametrize("name", ["pet_mini", "pet_tof_small", "ct_mini", "pet_stype1", "pet_stype2",
                                  "pet_stype4", "pet_stype5", "pet_odd_span1"])
def test_oracle_adjoint(name):
    o = make_options(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(5)
    s = min(1, g.n_subsets - 1)
    x = rng.random(g.n_img)
    y = rng.random(g.rays(s) * g.nbins)
    a = float(np.dot(orc.forward(g, x, s), y))
    b = float(np.dot(x, orc.backward(g, y, s)))
    assert a > 0 and abs(a - b) <= 1e-12 * abs(a)


def test_measurement_subsets_cover_sinogram_once():
    """Subset types 1/2/4/5: the union of all subsets' rays is every sinogram bin once."""
    for name in ["pet_stype1", "pet_stype2", "pet_stype4", "pet_stype5"]:
        o = make_options(name)
        g = orc.Geometry(o)
        full = make_options(name)
        full.subsets = 1
        full.subsetType = 8
        full.addProjector()
        gf = orc.Geometry(full)
        rng = np.random.default_rng(0)
        x = rng.random(g.n_img)
        y_full = orc.forward(gf, x, 0)
        got = np.concatenate([orc.forward(g, x, s) for s in range(g.n_subsets)])
        idx = np.asarray(o.index, dtype=np.int64)
        assert np.allclose(got, y_full[idx], rtol=1e-13, atol=0), name


def test_osem_loop_increases_loglik():
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(11)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    y = [rng.poisson(orc.forward(g, truth, s) * 10.0).astype(np.float64) for s in range(g.n_subsets)]
    x0 = np.ones(g.n_img)
    ll = []
    for it in (1, 2, 3):
        x = orc.osem(g, y, x0, it)
        ll.append(sum(orc.loglik(y[s], orc.forward(g, x, s), g.epps) for s in range(g.n_subsets)))
    assert ll[0] < ll[1] < ll[2]


def test_reference_cpu_library_agrees_when_built():
    """When oracle/_ref was built here, the live reference CPU projector
    reproduces the stored fixture (pins the fixture generation itself)."""
    if orc.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    p = load_golden("proj", "pet_mini")
    y = orc.ref_forward(g, p["image"].astype(np.float64), 0)
    assert orc.rel_l2(y, p["fp_0"]) < TOL
