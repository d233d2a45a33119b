"""Launch-shape tuning: every candidate shape computes the same projections
(parity with the FP64 oracle at 1e-5 relative L2 for each), the autotuner
returns a valid shape, and invalid shapes are rejected."""
import itertools

import numpy as np
import pytest

from conftest import make_options
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _init(name):
    o = make_options(name)
    o.initProj()
    return o


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


@pytest.mark.parametrize("name", ["ct_mini5", "ct_fine5"])
def test_bdd_every_shape_matches_oracle(cuda, name):
    o = _init(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(11)
    x = rng.uniform(0.0, 1.0, g.n_img)
    y = rng.uniform(0.0, 2.0, g.rays(0))
    ref_fp = orc.bdd_forward(g, x, 0)
    ref_bp, ref_s = orc.bdd_backward(g, y, 0, sens=True)
    from omega_b200 import _native
    shapes = [(c, z, r, 0) for c, z, r in itertools.product([8, 16], [4, 8, 16], [4, 8])]
    shapes += [(8, z, 4, 1) for z in (4, 8, 16)] + [(16, 16, 4, 1)]
    fps, bps = {}, {}
    for cols, zrun, rows, staged in shapes:
        o.tuning = {"bdd_fp_columns": cols, "bdd_bp_zrun": zrun, "bdd_fp_block_rows": rows,
                    "bdd_bp_block_rows": rows, "bdd_fp_staged": staged, "bdd_bp_staged": staged}
        fp = o.forwardProject(_t(x, cuda), 0).cpu().numpy()
        bp, s = o.backwardProject(_t(y, cuda), 0, sens=True)
        assert orc.rel_l2(fp, ref_fp) < TOL, (cols, rows, orc.rel_l2(fp, ref_fp))
        assert orc.rel_l2(bp.cpu().numpy(), ref_bp) < TOL, (zrun, rows, orc.rel_l2(bp.cpu().numpy(), ref_bp))
        assert orc.rel_l2(s.cpu().numpy(), ref_s) < TOL, (zrun, rows)
        fps[(cols, rows, staged)] = fp
        bps[(zrun, rows, staged)] = (bp.cpu().numpy(), s.cpu().numpy())
    assert _native.call("omb_take_device_error") == 0
    # staging the image / detector boxes in shared memory changes where the
    # data are read from, not the arithmetic
    for c in (8, 16):
        assert np.array_equal(fps[(c, 4, 1)].view(np.uint32), fps[(c, 4, 0)].view(np.uint32)), c
    for z in (8, 16):
        for a, b in zip(bps[(z, 4, 1)], bps[(z, 4, 0)]):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), z


def test_siddon_every_shape_matches_oracle(cuda):
    import ctypes

    import torch
    from omega_b200 import _native
    o = _init("pet_mini")
    g = orc.Geometry(o)
    n, m = g.n_img, o.measurementCount(-1)
    frames = 5
    rng = np.random.default_rng(12)
    imgs = rng.uniform(0.5, 2.0, (frames, n))
    ref = np.concatenate([orc.forward(g, imgs[0], s) for s in range(g.n_subsets)])
    ref_fp = [np.concatenate([orc.forward(g, imgs[f], s) for s in range(g.n_subsets)]) for f in range(frames)]
    assert orc.rel_l2(ref_fp[0], ref) == 0.0
    # backprojection of every frame over all subsets (measurements subset-contiguous)
    ys = rng.uniform(0.0, 2.0, (frames, m))
    ys[:, ::7] = 0.0
    cut = np.cumsum([0] + [g.rays(s) for s in range(g.n_subsets)])
    ref_bp = [sum(orc.backward(g, ys[f, cut[s]:cut[s + 1]], s) for s in range(g.n_subsets)) for f in range(frames)]
    X = _t(imgs, cuda)
    Yin = _t(ys, cuda)
    Y = torch.empty((frames, m), device=cuda)
    B = torch.empty((frames, n), device=cuda)
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    shapes = [(ps, fw, lay, 1) for ps, fw, lay in itertools.product([1, 2, 8, 16], [1, 2, 4, 8], [0, 1])]
    shapes += [(8, fw, lay, k) for fw, lay, k in itertools.product([1, 4, 8], [0, 1], [2, 4])]
    for ps, fw, lay, k in shapes:
        o.tuning = {"siddon_blocks_per_sm": ps, "siddon_frames_per_walk": fw, "siddon_frame_layout": lay,
                    "siddon_fp_steps": k}
        _native.call("omb_forward_frames", o._handle, -1, frames, ctypes.c_void_p(X.data_ptr()), n,
                     ctypes.c_void_p(Y.data_ptr()), m, st)
        B.fill_(-1.0)
        _native.call("omb_backward_frames", o._handle, -1, frames, ctypes.c_void_p(Yin.data_ptr()), m,
                     ctypes.c_void_p(B.data_ptr()), n, st)
        y, b = Y.cpu().numpy(), B.cpu().numpy()
        for f in range(frames):
            assert orc.rel_l2(y[f], ref_fp[f]) < TOL, (ps, fw, lay, k, f)
            assert orc.rel_l2(b[f], ref_bp[f]) < TOL, (ps, fw, lay, f, orc.rel_l2(b[f], ref_bp[f]))


@pytest.mark.parametrize("name,frames", [("ct_mini5", 1), ("pet_mini", 4)])
def test_autotune_returns_valid_shape(cuda, name, frames):
    o = _init(name)
    t = o.autotune(n_frames=frames, repeats=1)
    assert t == o.tuning
    assert 1 <= t["siddon_blocks_per_sm"] <= 32
    assert t["siddon_frames_per_walk"] in (1, 2, 4, 8)
    assert t["bdd_fp_columns"] in (8, 16)
    assert t["bdd_bp_zrun"] in (4, 8, 16)
    assert t["bdd_fp_block_rows"] in (4, 8) and t["bdd_bp_block_rows"] in (4, 8)
    assert t["siddon_frame_layout"] in (0, 1) and t["siddon_fp_steps"] in (1, 2, 4)
    g = orc.Geometry(o)
    x = np.random.default_rng(13).uniform(0.5, 1.5, g.n_img)
    fp = o.forwardProject(_t(x, cuda), 0).cpu().numpy()
    ref = orc.bdd_forward(g, x, 0) if name == "ct_mini5" else orc.forward(g, x, 0)
    assert orc.rel_l2(fp, ref) < TOL


@pytest.mark.parametrize("key,value", [("siddon_blocks_per_sm", 0), ("siddon_frames_per_walk", 3),
                                       ("bdd_fp_columns", 4), ("bdd_bp_zrun", 32),
                                       ("bdd_fp_block_rows", 2), ("bdd_bp_block_rows", 16),
                                       ("siddon_frame_layout", 2), ("siddon_fp_steps", 3)])
def test_invalid_shape_rejected(cuda, key, value):
    from omega_b200 import _native
    o = _init("ct_mini5")
    before = o.tuning
    with pytest.raises(_native.NativeError):
        o.tuning = {key: value}
    assert o.tuning == before
