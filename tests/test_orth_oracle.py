"""Projector types 2 (orthogonal distance) and 3 (volume of intersection):
the FP64 restatement pinned against the reference's own CPU projector
(oracle/_ref, projector_functions.h) in the restatement's CPU variant, the
type-3 volume table against the reference's computeVoxelVolumes
(tests/golden/vol_tables.npz), and properties of the GPU-kernel variant."""
import os
import warnings

import numpy as np
import pytest

from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
TUBES = {2: dict(tube_width_z=4.0, tube_width_xy=9.8), 3: dict(tube_radius=3.0)}


def _opts(base, pt, **kw):
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    cfg = dict(CONFIGS[base], projector_type=pt, subsets=1, subsetType=8)
    cfg.update(TUBES[pt])
    cfg.update(kw)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        o = apply(proj.projectorClass(), cfg)
        o.addProjector()
    return o


def _need_ref():
    if orc.ref_lib() is None:
        pytest.skip("oracle/_ref not built (needs the reference sources)")


@pytest.mark.parametrize("pt", [2, 3])
def test_cpu_variant_matches_reference_projector(pt):
    _need_ref()
    g = orc.Geometry(_opts("pet_mini", pt))
    g.cpu_mode = 1
    rng = np.random.default_rng(pt)
    img = rng.uniform(0.5, 1.5, g.n_img)
    a = orc.orth_forward(g, img, -1)
    r = orc.ref_orth(g, img, -1, True, pt)
    assert np.count_nonzero(a) > 0.9 * a.size
    assert orc.rel_l2(a, r) < 1e-12, orc.rel_l2(a, r)
    y = rng.uniform(0.0, 2.0, a.size)
    bi, bs = orc.orth_backward(g, y, -1, sens=True)
    ri, rs = orc.ref_orth(g, y, -1, False, pt, sens=True)
    assert orc.rel_l2(bi, ri) < 1e-12 and orc.rel_l2(bs, rs) < 1e-12


def test_cpu_variant_matches_reference_tof_type3():
    _need_ref()
    g = orc.Geometry(_opts("pet_mini_tof", 3))
    assert g.nbins == 7
    g.cpu_mode = 1
    rng = np.random.default_rng(7)
    img = rng.uniform(0.5, 1.5, g.n_img)
    a = orc.orth_forward(g, img, -1)
    assert orc.rel_l2(a, orc.ref_orth(g, img, -1, True, 3)) < 1e-12
    y = rng.uniform(0.0, 2.0, a.size)
    bi, bs = orc.orth_backward(g, y, -1, sens=True)
    ri, rs = orc.ref_orth(g, y, -1, False, 3, sens=True)
    assert orc.rel_l2(bi, ri) < 1e-12 and orc.rel_l2(bs, rs) < 1e-12


@pytest.mark.parametrize("pt", [2, 3])
def test_cpu_variant_matches_reference_with_corrections(pt):
    _need_ref()
    g = orc.Geometry(_opts("pet_mini", pt))
    g.cpu_mode = 1
    rng = np.random.default_rng(10 + pt)
    m = g.rays(-1)
    g.w = rng.uniform(0.5, 1.5, m)
    g.mu = rng.uniform(0.0, 0.01, g.n_img)
    img = rng.uniform(0.5, 1.5, g.n_img)
    a = orc.orth_forward(g, img, -1)
    assert orc.rel_l2(a, orc.ref_orth(g, img, -1, True, pt, norm=g.w, atten=g.mu)) < 1e-12
    y = rng.uniform(0.0, 2.0, m)
    bi = orc.orth_backward(g, y, -1)
    assert orc.rel_l2(bi, orc.ref_orth(g, y, -1, False, pt, norm=g.w, atten=g.mu)) < 1e-12


def test_volume_table_matches_reference():
    from omega_b200.projector import orth
    f = np.load(os.path.join(HERE, "golden", "vol_tables.npz"))
    cases = {"a": (1.0, 1.0, (2.0, 2.0, 2.5)), "b": (2.5, 1.0, (1.5, 1.5, 1.5))}

    class Opt:
        pass
    for tag, (R, r, d) in cases.items():
        o = Opt()
        o.tube_radius, o.voxel_radius = R, r
        o.dx, o.dy, o.dz = (np.array([v], dtype=np.float32) for v in d)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            orth.voxel_volumes(o)
        V, s = f["V_" + tag], f["s_" + tag]
        assert o.V.shape == V.shape and o.V.dtype == np.float32
        # bmin, bmax, Vmax and the scaled voxel radius as the reference sets them
        assert np.allclose([o.bmin, o.bmax, o.Vmax, o.voxel_radius], s, rtol=1e-12, atol=0)
        # the reference evaluates the closed form in float32, FP64 here: equal to float32 rounding
        assert np.max(np.abs(o.V.astype(np.float64) - V)) < 1e-6 * o.Vmax


@pytest.mark.parametrize("pt", [2, 3])
def test_kernel_variant_is_adjoint(pt):
    g = orc.Geometry(_opts("pet_mini", pt))
    rng = np.random.default_rng(20 + pt)
    x = rng.uniform(0.0, 1.0, g.n_img)
    y = rng.uniform(0.0, 1.0, g.rays(-1))
    ax = orc.orth_forward(g, x, -1)
    aty = orc.orth_backward(g, y, -1)
    lhs, rhs = float(np.dot(ax, y)), float(np.dot(x, aty))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


@pytest.mark.parametrize("pt", [2, 3])
def test_kernel_variant_scans_both_sides(pt):
    # the GPU kernel's descending in-slice scan adds the voxels on the other
    # side of the ray, so with a tube wider than a voxel its rays carry more
    # weight than the CPU variant's (type 3 also divides by L r^2 / pi
    # instead of L pi r^2)
    g = orc.Geometry(_opts("pet_mini", pt, **({"tube_width_z": 12.0} if pt == 2 else {"tube_radius": 6.0})))
    ones = np.ones(g.n_img)
    k = orc.orth_forward(g, ones, -1)
    g.cpu_mode = 1
    c = orc.orth_forward(g, ones, -1)
    if pt == 3:
        c = c * np.pi ** 2
    seen = c > 0
    assert np.median(k[seen] / c[seen]) > 1.05


def test_wider_tube_sees_more():
    a = orc.orth_forward(orc.Geometry(_opts("pet_mini", 2)), np.ones(32 * 32 * 15), -1)
    b = orc.orth_forward(orc.Geometry(_opts("pet_mini", 2, tube_width_z=8.0)), np.ones(32 * 32 * 15), -1)
    assert np.sum(b) > 1.5 * np.sum(a)
