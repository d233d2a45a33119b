"""Multi-rank host logic on CPU: two gloo ranks (127.0.0.1) check the frame
shares, the max-over-ranks timing reduction and the backprojection exchange
of a subset split across ranks (partial FP64 oracle backprojections summed by
all-reduce equal the whole subset's)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), here, os.path.join(here, "golden")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from conftest import make_options
        from omega_b200 import distributed as D
        from oracle import oracle as orc
        # frame shares and the timing reduction
        lo, hi = D.shard(24, rank, world)
        times = D.max_over_ranks([1.0 + rank, 5.0 - rank])
        # a subset's rays split across ranks by sinogram: each rank
        # backprojects its own sinograms, the all-reduce sums the parts
        o = make_options("pet_mini")
        g = orc.Geometry(o)
        s = 1
        n_sino = int(g.n_meas[s + 1] - g.n_meas[s])
        per = g.n_rows * g.n_cols
        y = np.random.default_rng(7).uniform(0.0, 2.0, g.rays(s))
        a, b = D.shard(n_sino, rank, world)
        part = y.copy()
        part[:a * per] = 0.0
        part[b * per:] = 0.0
        bp = orc.backward(g, part, s)
        yb = np.zeros_like(y)
        yb[a * per:b * per] = 1.0
        sens_part = orc.backward(g, yb, s)  # A^T 1 over this rank's rays
        tb, ts = torch.from_numpy(bp), torch.from_numpy(sens_part)
        D.allreduce_backprojection(tb, ts)
        full_bp = orc.backward(g, y, s)
        full_sens = orc.backward(g, np.ones_like(y), s)
        out.put((rank, (lo, hi), times, orc.rel_l2(tb.numpy(), full_bp), orc.rel_l2(ts.numpy(), full_sens)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, t0, e0, f0), (r1, s1, t1, e1, f1) = res
    assert s0 == (0, 12) and s1 == (12, 24)
    assert t0 == t1 == [2.0, 5.0]
    assert e0 < 1e-12 and e1 < 1e-12 and f0 < 1e-12 and f1 < 1e-12


@pytest.mark.parametrize("n,world", [(24, 5), (7, 3), (3, 4)])
def test_shares_cover_once(n, world):
    from omega_b200 import distributed as D
    covered = []
    for r in range(world):
        lo, hi = D.shard(n, r, world)
        covered.extend(range(lo, hi))
    assert covered == list(range(n))
