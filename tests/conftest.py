import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (REPO, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(kind, name):
    path = os.path.join(GOLDEN, f"{kind}_{name}.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def make_options(name):
    """Our projectorClass with the named option set, addProjector() done."""
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), CONFIGS[name] if name in CONFIGS else _extra(name))
    o.addProjector()
    return o


def listmode_events(base="pet_mini", n_events=4000, seed=0):
    """Seeded list-mode events on the LORs of a sinogram scanner: the
    (source, detector) coordinates of random sinogram bins, and the bins."""
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), dict(CONFIGS[base], subsets=1, subsetType=8))
    o.addProjector()
    xy = np.asarray(o.x, dtype=np.float32).reshape(-1, 4)
    z = np.asarray(o.z, dtype=np.float32).reshape(-1, 2)
    rng = np.random.default_rng(seed)
    b = rng.integers(0, xy.shape[0], n_events)
    k = rng.integers(0, z.shape[0], n_events)
    ev = np.stack([xy[b, 0], xy[b, 1], z[k, 0], xy[b, 2], xy[b, 3], z[k, 1]])  # 6 x events
    return o, ev, b + k * xy.shape[0]


def make_listmode_options(base="pet_mini", n_events=4000, event_seed=0, indexed=False, **extra):
    """projectorClass on list-mode (or index-based) events of a sinogram
    scanner, addProjector() done."""
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    _, ev, _ = listmode_events(base, n_events, event_seed)
    cfg = dict(CONFIGS[base])
    cfg.update(extra)
    o = apply(proj.projectorClass(), cfg)
    o.SinM = np.zeros(n_events, dtype=np.float32)
    if indexed:
        pts = np.concatenate([ev[[0, 1]].T, ev[[3, 4]].T])
        table, inv = np.unique(pts, axis=0, return_inverse=True)
        zt, zinv = np.unique(np.concatenate([ev[2], ev[5]]), return_inverse=True)
        o.useIndexBasedReconstruction = True
        o.x = table.astype(np.float32).ravel()          # [x, y] per crystal
        o.z = zt.astype(np.float32)
        o.trIndex = np.stack([inv[:n_events], inv[n_events:]]).astype(np.uint16)
        o.axIndex = np.stack([zinv[:n_events], zinv[n_events:]]).astype(np.uint16)
    else:
        o.x = np.asfortranarray(ev)
    o.addProjector()
    return o


def _extra(name):
    from make_golden import CONFIGS_EXTRA
    return CONFIGS_EXTRA[name]


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from omega_b200 import _native
    _native.lib()
    return torch.device("cuda:0")
