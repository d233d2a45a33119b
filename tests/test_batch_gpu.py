"""Batches of independent CT reconstructions in one persistent launch
(omb_batch_*): every item's projection equals the item projected on its own
(and the FP64 oracle), for fan-beam slices of different image sizes and view
counts."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
SIZES = [(64, 90), (96, 60), (48, 120), (80, 45), (32, 30)]


def _items():
    from omega_b200.projector.batch import fanbeam_slice
    return [fanbeam_slice(n, v) for n, v in SIZES]


def test_batch_matches_single_items_and_oracle(cuda):
    import torch
    from omega_b200.projector.batch import ProjectorBatch
    items = _items()
    batch = ProjectorBatch(items)
    rng = np.random.default_rng(21)
    imgs = [rng.uniform(0.0, 1.0, int(o.N[0])) for o in items]
    ys = [rng.uniform(0.0, 2.0, o.nRowsD * o.nColsD * o.nProjections) for o in items]
    x = torch.tensor(np.concatenate(imgs), dtype=torch.float32, device=cuda)
    yin = torch.tensor(np.concatenate(ys), dtype=torch.float32, device=cuda)
    fp = batch.forward(x).cpu().numpy()
    bp = batch.backward(yin).cpu().numpy()
    io, mo = batch.image_offsets, batch.measurement_offsets
    for i, o in enumerate(items):
        o.initProj()
        g = orc.Geometry(o)
        xi = torch.tensor(imgs[i], dtype=torch.float32, device=cuda)
        yi = torch.tensor(ys[i], dtype=torch.float32, device=cuda)
        single_fp = o.forwardProject(xi, -1).cpu().numpy()
        single_bp = o.backwardProject(yi, -1).cpu().numpy()
        assert orc.rel_l2(fp[mo[i]:mo[i + 1]], single_fp) < 1e-6, i
        assert orc.rel_l2(bp[io[i]:io[i + 1]], single_bp) < 1e-6, i
        assert orc.rel_l2(fp[mo[i]:mo[i + 1]], orc.forward(g, imgs[i], -1)) < 1e-5, i
        assert orc.rel_l2(bp[io[i]:io[i + 1]], orc.backward(g, ys[i], -1)) < 1e-5, i


def test_batch_rejects_unsupported_items(cuda):
    from configs import CONFIGS, apply
    from omega_b200 import _native
    from omega_b200.projector import proj
    from omega_b200.projector.batch import ProjectorBatch
    pet = apply(proj.projectorClass(), CONFIGS["pet_mini"])
    pet.addProjector()
    with pytest.raises(_native.NativeError):
        ProjectorBatch(_items()[:1] + [pet])
