"""List-mode and index-based event data: the FP64 oracle against the
reference's own CPU projector run in list-mode (get_detector_coordinates_raw,
projector_functions.h:357-368), and against the sinogram oracle on the same
LORs.  CPU only."""
import numpy as np
import pytest

from conftest import listmode_events, make_listmode_options
from oracle import oracle as orc

TOL = 1e-12


@pytest.mark.skipif(orc.ref_lib() is None, reason="reference CPU projector not built")
@pytest.mark.parametrize("subset_type", [0, 1, 3])
def test_listmode_oracle_matches_reference(subset_type):
    o = make_listmode_options(subsets=3, subsetType=subset_type, event_seed=1)
    assert o.listmode == 1 and int(o.nRowsD) == 1
    g = orc.Geometry(o)
    rng = np.random.default_rng(2)
    x = rng.uniform(0.5, 2.0, g.n_img)
    for s in range(3):
        assert orc.rel_l2(orc.forward(g, x, s), orc.ref_listmode(g, x, s, True)) < TOL
        y = rng.uniform(0.0, 2.0, g.rays(s))
        bp, sens = orc.backward(g, y, s, sens=True)
        ref_bp, ref_s = orc.ref_listmode(g, y, s, False, sens=True)
        assert orc.rel_l2(bp, ref_bp) < TOL and orc.rel_l2(sens, ref_s) < TOL


def test_listmode_subsets_follow_the_reference_split():
    """Type 0: contiguous blocks, the last one takes the remainder; type 1:
    every 3rd event; type 3: a seeded permutation whose last block drops the
    final event, as indices.py:107-126 does."""
    o = make_listmode_options(subsets=3, subsetType=0, event_seed=1)
    assert list(np.diff(o.nMeas)) == [1333, 1333, 1334]
    o = make_listmode_options(subsets=3, subsetType=1, event_seed=1)
    assert list(np.diff(o.nMeas)) == [1334, 1333, 1333]
    assert np.array_equal(o.index[:3], [0, 3, 6])
    o = make_listmode_options(subsets=3, subsetType=3, event_seed=1, seed=5)
    assert int(o.nMeas[-1]) == 3999 and o.index.size == 3999


def test_events_equal_sinogram_bins_and_indices():
    o0, ev, bins = listmode_events(seed=1)
    g0 = orc.Geometry(o0)
    g = orc.Geometry(make_listmode_options(subsets=1, event_seed=1))
    gi = orc.Geometry(make_listmode_options(subsets=1, event_seed=1, indexed=True))
    x = np.random.default_rng(2).uniform(0.5, 2.0, g.n_img)
    y = orc.forward(g, x, -1)
    assert np.array_equal(y, orc.forward(g0, x, -1)[bins])
    assert np.array_equal(orc.forward(gi, x, -1), y)
