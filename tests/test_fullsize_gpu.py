"""Full-size workloads of the benchmark configurations, checked against the
FP64 oracle where the oracle finishes in seconds and through size-independent
properties where it does not:
  * the CPU-runnable PET OSEM workload (288 crystals x 16 rings, 144 x 144 x
    31 sinograms, 64 x 64 x 16 image, 8 subsets, 1e7 counts): 2 OSEM
    iterations (CUDA-graph replay) against the oracle's OSEM loop;
  * the precision workload (672 crystals x 55 rings, 400 x 336 x 109
    sinograms, 15 TOF bins of 200 ps FWHM, 200 x 200 x 109 image, projector
    type 4, 16 subsets): BF16 image reads against the FP64 oracle on one subset (the
    stated error), the int64 fixed-point TOF backprojection bit-identical run
    to run, and the float backprojection within 1e-5 of it."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _cylinder_phantom(g, seed):
    rng = np.random.default_rng(seed)
    xs = (np.arange(g.nx) + 0.5) * g.d[0] + g.b[0]
    zs = (np.arange(g.nz) + 0.5) * g.d[2] + g.b[2]
    X, Y, Z = np.meshgrid(xs, xs, zs, indexing="ij")
    r = 0.8 * abs(g.b[0])
    img = ((X ** 2 + Y ** 2) < r * r).astype(np.float64)
    for k in range(5):
        c = rng.uniform(-0.5 * r, 0.5 * r, 2)
        rad = rng.uniform(0.08, 0.15) * r
        img[((X - c[0]) ** 2 + (Y - c[1]) ** 2) < rad * rad] = 4.0 if k < 4 else 0.0
    return img.ravel(order="F")


def test_cfg0_osem_two_iterations_match_oracle(cuda):
    from configs import CONFIGS, apply
    from omega_b200 import reconstruction as rec
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), CONFIGS["pet_cfg0"])
    o.addProjector()
    o.initProj()
    g = orc.Geometry(o)
    truth = _cylinder_phantom(g, 3)
    clean = [orc.forward(g, truth, s) for s in range(g.n_subsets)]
    scale = 1e7 / sum(c.sum() for c in clean)
    rng = np.random.default_rng(4)
    ys = [rng.poisson(c * scale).astype(np.float32) for c in clean]
    x = rec.OSEM(o, np.concatenate(ys)).iterate(2, use_graph=True).cpu().numpy()
    ref = orc.osem(g, ys, np.ones(g.n_img), 2)
    assert orc.rel_l2(x, ref) < 5e-5, orc.rel_l2(x, ref)


def _precision_options(**extra):
    from configs import _pet, apply
    from omega_b200.projector import proj
    c = 2.99792458e11  # mm/s
    width = 848.0 / 15 / (c / 2)   # 15 bins covering +-424 mm (the FOV diagonal)
    cfg = _pet(42, 16, 55, 856, 400, 336, 200, 109, 600, 436, subsets=16, NSinos=109, TOF_bins=15,
               TOF_bins_used=15, TOF_FWHM=200e-12, TOF_width=width, projector_type=4)
    cfg["TotSinos"] = int(np.sum(__import__("configs")._segments(55, 3, 54, 109)))
    cfg.update(extra)
    o = apply(proj.projectorClass(), cfg)
    o.addProjector()
    o.initProj()
    return o


def test_precision_workload_bf16_error_and_int64_determinism(cuda):
    import torch
    o16 = _precision_options(imageReadPrecision="bf16")
    g = orc.Geometry(o16)
    assert g.nbins == 15 and (g.nx, g.ny, g.nz) == (200, 200, 109)
    assert g.rays(-1) == 400 * 336 * 109
    # values off the BF16 grid (0, 1 and 4 are exact in BF16)
    x = _cylinder_phantom(g, 7) * 1.2345 + 0.1 * np.random.default_rng(8).random(g.n_img)
    # BF16 reads against the FP64 oracle on subset 0 (one sixteenth of the rays)
    y16 = o16.forwardProject(_t(x, cuda), 0).cpu().numpy()
    err = orc.rel_l2(y16, orc.interp_forward(g, x, 0))
    assert 1e-6 < err < 4e-3, err
    del o16
    # int64 fixed-point TOF backprojection of all 219.7 M bins: bit-identical
    # (one subset: backwardProject(y, -1) means "the object's current subset",
    # as in the reference)
    o64 = _precision_options(use_64bit_atomics=True, subsets=1)
    m = o64.measurementCount(0)
    assert m == 400 * 336 * 109 * 15
    y = torch.rand(m, generator=torch.Generator(device=cuda).manual_seed(5), device=cuda)
    a = o64.backwardProject(y, 0).cpu().numpy()
    b = o64.backwardProject(y, 0).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    o64.use_64bit_atomics = False
    f = o64.backwardProject(y, 0).cpu().numpy()
    assert orc.rel_l2(f, a) < 1e-5
