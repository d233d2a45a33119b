"""Geometry and subset ordering of our projectorClass vs the reference's own
addProjector() output (golden fixtures made by tests/golden/make_golden.py).
Everything here must match bit for bit."""
import numpy as np
import pytest

from conftest import load_golden, make_options
from configs import CONFIGS, GEOMETRY_KEYS, SCALAR_KEYS

NAMES = list(CONFIGS) + ["pet_tof_small"]


@pytest.mark.parametrize("name", NAMES)
def test_geometry_bit_exact(name):
    g = load_golden("geom", name)
    o = make_options(name)
    for k in GEOMETRY_KEYS:
        ours = np.asarray(getattr(o, k))
        ref = g[k]
        assert ours.dtype == ref.dtype, (k, ours.dtype, ref.dtype)
        assert ours.shape == ref.shape, (k, ours.shape, ref.shape)
        assert np.array_equal(ours, ref), f"{name}: {k} differs"
    for k in SCALAR_KEYS:
        ours = np.asarray(getattr(o, k))
        assert np.array_equal(ours, g["s_" + k]), f"{name}: {k} {ours} != {g['s_' + k]}"
    for k in [k for k in g if k.startswith("p_")]:
        ours = np.asarray(getattr(o, k[2:]))
        assert ours.dtype == g[k].dtype and np.array_equal(ours, g[k]), f"{name}: {k[2:]} {ours} != {g[k]}"
    if "TOFCenter" in g:
        assert np.array_equal(np.asarray(o.TOFCenter), g["TOFCenter"])
    if "uV" in g:
        assert np.array_equal(np.asarray(o.uV), g["uV"])


def test_cfg0_subset_order():
    o = make_options("pet_cfg0")
    assert o.index.tolist()[:12] == [0, 8, 16, 24, 1, 9, 17, 25, 2, 10, 18, 26]
    assert o.nMeas.tolist() == [0, 4, 8, 12, 16, 20, 24, 28, 31]
    assert o.nProjSubset.ravel().tolist() == [4, 4, 4, 4, 4, 4, 4, 3]
    assert int(o.nTotMeas[-1]) == 144 * 144 * 31


def test_error_checks_match_reference_messages():
    from configs import apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), CONFIGS["pet_mini"])
    o.span = 4
    with pytest.raises(ValueError, match="Span value has to be odd and positive"):
        o.addProjector()
    o = apply(proj.projectorClass(), CONFIGS["pet_mini"])
    o.Nang = 80
    with pytest.raises(ValueError, match="Number of sinogram angles can be at most"):
        o.addProjector()
    o = apply(proj.projectorClass(), CONFIGS["pet_mini"])
    o.projector_type = 5
    with pytest.raises(ValueError, match="Projector type 5 is only supported with CT data"):
        o.addProjector()
    o = apply(proj.projectorClass(), CONFIGS["pet_mini_tof"])
    o.TOF_FWHM = 0.
    with pytest.raises(ValueError, match="TOF FWHM"):
        o.addProjector()


def test_measurement_reorder_matches_parse_inputs():
    """parseInputs (prepass.py:346-352): SinM[:, :, index] for subset types >= 8."""
    o = make_options("pet_mini")
    rng = np.random.default_rng(3)
    sino = rng.random((o.nRowsD, o.nColsD, o.nProjections)).astype(np.float32)
    o.SinM = sino.copy()
    o._parse_inputs()
    assert np.array_equal(o.SinM, sino[:, :, o.index])
