"""PET corrections of the type-1 projector (normalisation, multiplicative
scatter, attenuation as an image or as per-LOR factors): the FP64 oracle
restatement against the reference's own CPU projector
(projectorType123Implementation4, projector_functions.h:1754-1832) run with
the same corrections.  CPU only; skipped when oracle/_ref was not built."""
import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

pytestmark = pytest.mark.skipif(orc.ref_lib() is None, reason="reference CPU projector not built")
TOL = 1e-12


def _setup(name, seed):
    o = make_options(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.5, 2.0, g.n_img)
    total = int(g.n_meas[-1]) if g.meas_level() else g.rays(-1)
    w = rng.uniform(0.5, 1.5, total)
    # water-like attenuation with structure: 0.0096 / mm +- 50 %
    mu = 0.0096 * rng.uniform(0.5, 1.5, g.n_img)
    return g, rng, x, w, mu


def _span(g, subset):
    off = int(g.n_meas[subset]) * g.n_rows * g.n_cols
    return off, off + g.rays(subset)


@pytest.mark.parametrize("name", ["pet_mini", "pet_mini_tof"])
def test_norm_and_attenuation_image_match_reference(name):
    g, rng, x, w, mu = _setup(name, 1)
    for subset in range(g.n_subsets):
        a, b = _span(g, subset)
        g.w, g.mu = w, mu
        fp = orc.forward(g, x, subset)
        y = rng.uniform(0.0, 2.0, g.rays(subset) * g.nbins)
        bp, sens = orc.backward(g, y, subset, sens=True)
        g.w = g.mu = None
        ref_fp = orc.ref_corrected(g, x, subset, True, norm=w[a:b], atten=mu)
        ref_bp, ref_s = orc.ref_corrected(g, y, subset, False, norm=w[a:b], atten=mu, sens=True)
        assert orc.rel_l2(fp, ref_fp) < TOL, subset
        assert orc.rel_l2(bp, ref_bp) < TOL, subset
        assert orc.rel_l2(sens, ref_s) < TOL, subset
        # the corrections matter: the uncorrected projection is far off
        assert orc.rel_l2(orc.forward(g, x, subset), ref_fp) > 0.5


def test_lor_attenuation_and_scatter_as_weights():
    """ATNM and SCATTER are per-measurement multipliers: their product with
    the normalisation is the one weight the projector takes."""
    g, rng, x, w, mu = _setup("pet_mini", 2)
    subset = 1
    a, b = _span(g, subset)
    att = rng.uniform(0.3, 1.0, b - a)
    sc = rng.uniform(0.8, 1.2, b - a)
    g.w = np.ones(w.size)
    g.w[a:b] = w[a:b] * att * sc
    fp = orc.forward(g, x, subset)
    g.w = None
    ref = orc.ref_corrected(g, x, subset, True, norm=w[a:b], atten=att, ct_atten=False, scat=sc)
    assert orc.rel_l2(fp, ref) < TOL


def test_corrected_pair_is_adjoint():
    g, rng, x, w, mu = _setup("pet_stype1", 3)
    g.w, g.mu = w, mu
    s = 1
    y = rng.random(g.rays(s))
    lhs = float(np.dot(orc.forward(g, x, s), y))
    rhs = float(np.dot(x, orc.backward(g, y, s)))
    assert lhs > 0 and abs(lhs - rhs) <= 1e-12 * abs(lhs)
