"""CPU checks of the type-5 restatements: the ray-driven (scatter)
backprojection is the exact adjoint of the forward projection, which the
reference's kernels pin (tests/test_refcl_pin.py), and its sensitivity is
A^T 1; the reference's voxel-driven gather is close to it but not equal."""
import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc


@pytest.mark.parametrize("name", ["ct_mini5", "ct_fine5"])
def test_ray_backprojection_is_the_adjoint(name):
    o = make_options(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(31)
    x = rng.uniform(0.0, 1.0, g.n_img)
    y = rng.uniform(0.0, 1.0, g.rays(0))
    fx = orc.bdd_forward(g, x, 0)
    bt, sens = orc.bdd_backward_ray(g, y, 0, sens=True)
    a, b = float(np.dot(fx, y)), float(np.dot(x, bt))
    assert abs(a - b) <= 1e-12 * abs(a)
    assert orc.rel_l2(sens, orc.bdd_backward_ray(g, np.ones_like(y), 0)) < 1e-14
    # the gather of the reference is a different (nearly adjoint) operator
    c = float(np.dot(x, orc.bdd_backward(g, y, 0)))
    assert 1e-8 < abs(a - c) / abs(a) < 1e-2
