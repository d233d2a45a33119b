"""List-mode (6 coordinates per event) and index-based (crystal / ring index
pairs) event data through the type-1 and type-4 kernels: CUDA against the
FP64 oracle (pinned to the reference CPU projector in list-mode by
test_listmode_oracle.py), events bit-identical to the sinogram bins they
sample, index-based bit-identical to list-mode, corrections per event."""
import numpy as np
import pytest

from conftest import listmode_events, make_listmode_options, make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


@pytest.mark.parametrize("subset_type", [0, 1, 3])
@pytest.mark.parametrize("indexed", [False, True])
def test_events_match_oracle(cuda, subset_type, indexed):
    o = make_listmode_options(subsets=3, subsetType=subset_type, event_seed=2, indexed=indexed)
    o.initProj()
    g = orc.Geometry(o)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.5, 2.0, g.n_img)
    for s in range(3):
        fp = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        assert orc.rel_l2(fp, orc.forward(g, x, s)) < TOL, s
        y = rng.uniform(0.0, 2.0, g.rays(s))
        bp, sens = o.backwardProject(_t(y, cuda), s, sens=True)
        ref_bp, ref_s = orc.backward(g, y, s, sens=True)
        assert orc.rel_l2(bp.cpu().numpy(), ref_bp) < TOL, s
        assert orc.rel_l2(sens.cpu().numpy(), ref_s) < TOL, s


def test_events_equal_their_sinogram_bins(cuda):
    o_sino, ev, bins = listmode_events(seed=4)
    o_sino.initProj()
    o = make_listmode_options(subsets=1, event_seed=4)
    o.initProj()
    oi = make_listmode_options(subsets=1, event_seed=4, indexed=True)
    oi.initProj()
    x = _t(np.random.default_rng(5).uniform(0.5, 2.0, int(np.ravel(o.N)[0])), cuda)
    y_sino = o_sino.forwardProject(x, 0).cpu().numpy()
    y = o.forwardProject(x, 0).cpu().numpy()
    yi = oi.forwardProject(x, 0).cpu().numpy()
    assert np.array_equal(y.view(np.uint32), y_sino[bins].view(np.uint32))
    assert np.array_equal(yi.view(np.uint32), y.view(np.uint32))
    e = _t(np.random.default_rng(6).uniform(0.0, 2.0, y.size), cuda)
    b = o.backwardProject(e, 0).cpu().numpy()
    bi = oi.backwardProject(e, 0).cpu().numpy()
    assert orc.rel_l2(bi, b) < 1e-6


def test_events_type4_and_corrections(cuda):
    # projector type 4 on events
    o = make_listmode_options(subsets=2, subsetType=1, event_seed=7, projector_type=4)
    o.initProj()
    g = orc.Geometry(o)
    x = np.random.default_rng(8).uniform(0.5, 2.0, g.n_img)
    for s in range(2):
        fp = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        assert orc.rel_l2(fp, orc.interp_forward(g, x, s)) < TOL, s
    # normalisation per event and an attenuation image, type 1
    o = make_listmode_options(subsets=2, subsetType=1, event_seed=9)
    rng = np.random.default_rng(10)
    n_ev = int(np.ravel(o.nTotMeas)[-1])
    o.normalization_correction = 1
    o.normalization = rng.uniform(0.5, 1.5, n_ev).astype(np.float32)
    o.attenuation_correction = 1
    o.vaimennus = (0.0096 * rng.uniform(0.5, 1.5, int(np.ravel(o.N)[0]))).astype(np.float32)
    o.initProj()
    g = orc.Geometry(o)
    g.w = o.normalization.astype(np.float64)
    g.mu = o.vaimennus.astype(np.float64)
    for s in range(2):
        fp = o.forwardProject(_t(x, cuda), s).cpu().numpy()
        assert orc.rel_l2(fp, orc.forward(g, x, s)) < TOL, s
        y = rng.uniform(0.0, 2.0, g.rays(s))
        assert orc.rel_l2(o.backwardProject(_t(y, cuda), s).cpu().numpy(), orc.backward(g, y, s)) < TOL, s


def test_index_out_of_range_rejected(cuda):
    from omega_b200 import _native
    o = make_listmode_options(subsets=1, event_seed=11, indexed=True)
    o.trIndex = o.trIndex.copy()
    o.trIndex[5] = 60000
    with pytest.raises(_native.NativeError):
        o.initProj()
