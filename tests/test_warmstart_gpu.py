"""What the trained warm-start network gains, on held-out studies.

The committed weights (omega_b200/weights/warmstart_pet128.npz, trained on
seeds 1,000,000-1,004,999) on two studies never seen in training or in the
committed evaluation (seeds 4,000,000 and 4,000,001), dynamic-PET scanner,
16 subsets:
  * the warm path -- 2 OSEM iterations, the network, at most 4 more
    iterations -- reaches the log-likelihood plain OSEM has after 20
    iterations (L20);
  * plain OSEM with the same 6 iterations but no network stays below L20;
  * the warm path, timed with a fixed 4-iteration continuation and its
    log-likelihood check inside the timed region, takes under half the
    plain 20 iterations' time.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "omega_b200", "weights",
                       "warmstart_pet128.npz")


def test_warm_start_gain_on_held_out_studies(cuda):
    import torch
    from omega_b200 import reconstruction as rec
    from omega_b200 import warmstart as ws
    state = dict(np.load(WEIGHTS))
    o = ws.pet_geometry()
    o.initProj()
    seed, n = 4_000_000, 2
    summary, rows = ws.evaluate(o, state, seed, n, (1e7, 1e8), converged=20, batch=n, timing_studies=n)
    assert all(r["k"] is not None and r["k"] <= 4 for r in rows), [r["k"] for r in rows]
    assert summary["timed_reached_L20"] == n
    assert summary["time_ratio_median"] < 0.5, summary["time_ratio_median"]
    # the same number of iterations without the network falls short of L20
    N = int(o.N[0])
    truth = ws.phantoms(o, seed, n, cuda)
    m = ws.simulate(o, truth, [r["counts"] for r in rows], seed)
    plain = rec.OSEMBatch(o, m, x0=np.ones(N, dtype=np.float32))
    plain.iterate(6, use_graph=True)
    work = torch.empty(n * o.measurementCount(-1), device=cuda)
    L6 = ws.loglik_frames(o, plain.x, m, work)
    assert all(L6[f] < rows[f]["L20"] for f in range(n)), (L6, [r["L20"] for r in rows])
