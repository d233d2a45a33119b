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
