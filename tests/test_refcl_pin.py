"""The FP64 restatements of projector types 4 and 5, the TV gradient and the
PDHG update against the reference's own kernel sources run on the host.

oracle/_ref/libref_cl_*.so are OMEGA's projectorType5.cl, projectorType4.cl
and auxKernels.cl compiled unchanged with g++ through oracle/cl_host_shim.h
(built by oracle/Makefile when the OMEGA sources are given).  In FP64 with
exact texture weights and unrounded scale scalars they compute the
reference's algorithm without its single-precision rounding, and the
restatements the GPU kernels are tested against must equal them to rounding.
The same kernels in FP32 with 8-bit texture weights (the reference's GPU
arithmetic) are compared too, to state the reference's own error.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, os.path.dirname(HERE))

from configs import CONFIGS, apply  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from oracle import ref_cl  # noqa: E402

pytestmark = pytest.mark.skipif(not ref_cl.available(), reason="oracle/_ref not built (needs the OMEGA sources)")

# restatement vs reference, both FP64 with the same inputs
PIN = 1e-11


def _proj(name, **extra):
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), dict(CONFIGS[name], **extra))
    o.addProjector()
    return o


# ---------------------------------------------------------------------------
# projector type 5 (branchless distance-driven)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name", ["ct_mini5", "ct_fine5", "ct_cfg1_4v"])
def test_bdd_forward_pinned(name):
    o = _proj(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(11)
    x = rng.uniform(0.0, 0.02, g.n_img)
    ours = orc.bdd_forward(g, x, -1)
    ref = ref_cl.RefCT(o, exact_inputs=True).bdd_forward(x, -1)
    assert orc.rel_l2(ours, ref) < PIN
    # with the float32 scale scalars the reference's launch passes
    ref32in = ref_cl.RefCT(o).bdd_forward(x, -1)
    assert orc.rel_l2(ours, ref32in) < 1e-6
    if name != "ct_cfg1_4v":
        # the reference's own GPU arithmetic (FP32, 8-bit texture weights)
        gpu_like = ref_cl.RefCT(o).bdd_forward(x, -1, precision="f")
        assert orc.rel_l2(gpu_like, ref) < 5e-3


@pytest.mark.parametrize("name", ["ct_fine5", "ct_cfg1_4v"])
def test_bdd_backward_pinned(name):
    """Panels that cover every voxel footprint: image and sensitivity equal."""
    o = _proj(name)
    g = orc.Geometry(o)
    rng = np.random.default_rng(12)
    y = rng.uniform(0.0, 1.0, g.rays(-1))
    ours, sens = orc.bdd_backward(g, y, -1, sens=True)
    ref, rsens = ref_cl.RefCT(o, exact_inputs=True).bdd_backward(y, -1, sens=True)
    assert orc.rel_l2(ours, ref) < PIN
    assert orc.rel_l2(sens, rsens) < PIN


def test_bdd_backward_off_panel():
    """ct_mini5's panel does not cover the volume: footprints beyond the far
    panel edge read the clamped last summed-area node four times, and the
    reference's `apu != 0` test then sees the rounding residue of
    A + D - C - B, so it adds those views to the sensitivity (and a residue to
    the image).  The restatement counts them as zero, as exact arithmetic
    does: the images agree to rounding, and the reference's sensitivity only
    ever has extra views."""
    o = _proj("ct_mini5")
    g = orc.Geometry(o)
    rng = np.random.default_rng(13)
    y = rng.uniform(0.0, 1.0, g.rays(-1))
    ours, sens = orc.bdd_backward(g, y, -1, sens=True)
    ref, rsens = ref_cl.RefCT(o, exact_inputs=True).bdd_backward(y, -1, sens=True)
    assert orc.rel_l2(ours, ref) < PIN
    assert np.all(rsens >= sens - 1e-9 * sens.max())
    assert np.count_nonzero(rsens > sens + 1e-9 * sens.max()) > 0


# ---------------------------------------------------------------------------
# projector type 4 (interpolation)
# ---------------------------------------------------------------------------

# A FOV that is not a multiple of the crystal pitch: no sample of the PET
# type-4 backprojection falls exactly on a voxel face.
OFFSET_FOV = dict(FOVa_x=180.37, FOVa_y=180.37, axial_fov=33.71)


@pytest.mark.parametrize("name,extra", [("pet_mini4", {}), ("pet_mini4", OFFSET_FOV),
                                        ("pet_mini4_tof", OFFSET_FOV), ("ct_mini4", {})])
def test_interp_forward_pinned(name, extra):
    o = _proj(name, **extra)
    g = orc.Geometry(o)
    R = ref_cl.RefCT(o, exact_inputs=True) if o.CT else ref_cl.RefPET(o, exact_inputs=True)
    rng = np.random.default_rng(14)
    x = rng.uniform(0.5, 1.5, g.n_img)
    for s in (0, 1):
        ours = orc.interp_forward(g, x, s)
        assert orc.rel_l2(ours, R.interp_forward(x, s)) < PIN
        gpu_like = (ref_cl.RefCT(o) if o.CT else ref_cl.RefPET(o)).interp_forward(x, s, precision="f")
        assert orc.rel_l2(gpu_like, ours) < 5e-3


@pytest.mark.parametrize("name,extra", [("pet_mini4", OFFSET_FOV), ("pet_mini4_tof", OFFSET_FOV), ("ct_mini4", {})])
def test_interp_backward_pinned(name, extra):
    o = _proj(name, **extra)
    g = orc.Geometry(o)
    R = ref_cl.RefCT(o, exact_inputs=True) if o.CT else ref_cl.RefPET(o, exact_inputs=True)
    rng = np.random.default_rng(15)
    for s in (0, 1):
        y = rng.uniform(0.0, 1.0, R.interp_forward(np.zeros(g.n_img), s).size)
        back = orc.interp_ct_backward if o.CT else orc.interp_backward
        ours, sens = back(g, y, s, sens=True)
        ref, rsens = R.interp_backward(y, s, sens=True)
        assert orc.rel_l2(ours, ref) < PIN
        assert orc.rel_l2(sens, rsens) < PIN


def test_interp_backward_face_samples():
    """With a FOV of whole crystal pitches, axis-parallel PET rays sample
    exactly on voxel faces and the nearest-voxel choice floor(p N) is decided
    by rounding: the reference's own FP32 and FP64 runs differ there by a few
    1e-3, and the restatement (FP64 decision) sits within that spread."""
    o = _proj("pet_mini4")
    g = orc.Geometry(o)
    R = ref_cl.RefPET(o, exact_inputs=True)
    rng = np.random.default_rng(16)
    y = rng.uniform(0.0, 1.0, g.rays(0))
    ours = orc.interp_backward(g, y, 0)
    ref64 = R.interp_backward(y, 0)
    ref32 = ref_cl.RefPET(o).interp_backward(y, 0, precision="f")
    spread = orc.rel_l2(ref32, ref64)
    assert 1e-4 < spread < 1e-2
    assert orc.rel_l2(ours, ref64) < 2 * spread


# ---------------------------------------------------------------------------
# TV gradient and PDHG update
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("shape", [(17, 13, 9), (32, 32, 24)])
@pytest.mark.parametrize("smooth", [1e-2, 1e-4])
def test_tv_gradient_pinned(shape, smooth):
    rng = np.random.default_rng(17)
    u = rng.uniform(0.0, 1.0, int(np.prod(shape)))
    ours = orc.tv_gradient(u, shape, smooth, 0.7)
    ref = ref_cl.tv_gradient(u, shape, smooth, 0.7, exact_inputs=True)
    assert orc.rel_l2(ours, ref) < 1e-13
    ref32 = ref_cl.tv_gradient(u, shape, smooth, 0.7, precision="f")
    assert orc.rel_l2(ours, ref32) < 1e-5


def test_pdhg_update_pinned():
    """One PDHG primal step of the restatement (oracle.pdhg_tv's update) equals
    auxKernels.cl PDHGUpdate, with the clamp active on part of the image."""
    shape = (20, 18, 7)
    rng = np.random.default_rng(18)
    n = int(np.prod(shape))
    im, u = rng.uniform(0, 1, n), rng.uniform(0, 1, n)
    rhs = rng.normal(0, 2, n)
    tau, theta, eps = 0.3, 1.0, 1e-5
    u_new = np.maximum(eps, u - tau * rhs)
    x_new = u_new + theta * (u_new - u)
    assert np.any(u - tau * rhs < eps)
    ref_x, ref_u = ref_cl.pdhg_update(im, rhs, u, shape, tau, theta, eps, exact_inputs=True)
    assert orc.rel_l2(x_new, ref_x) < 1e-15
    assert orc.rel_l2(u_new, ref_u) < 1e-15


def test_pdhg_iteration_pinned():
    """Two PDHG+TV iterations of oracle.pdhg_tv against the same loop built
    from the reference's kernels: its type-5 projector pair, TVKernel and
    PDHGUpdate (dual step computeForwardProject.h:227-316)."""
    o = _proj("ct_fine5")
    g = orc.Geometry(o)
    R = ref_cl.RefCT(o, exact_inputs=True)
    shape = (g.nx, g.ny, g.nz)
    rng = np.random.default_rng(19)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    y = orc.bdd_forward(g, truth, -1)
    x0 = np.full(g.n_img, 1e-3)
    tau, beta, smooth, sigma = 1e-4, 0.01, 1e-4, 1.0
    ours = orc.pdhg_tv(g, y, x0, 2, tau, beta, smooth, sigma=sigma)
    x, u = x0.copy(), x0.copy()
    p = np.zeros(g.rays(-1))
    for _ in range(2):
        p = (p + sigma * (R.bdd_forward(x, -1) - y)) / (1.0 + sigma)
        rhs = R.bdd_backward(p, -1) + ref_cl.tv_gradient(x, shape, smooth, beta, exact_inputs=True)
        x, u = ref_cl.pdhg_update(x, rhs, u, shape, tau, 1.0, 1e-5, exact_inputs=True)
    assert orc.rel_l2(ours, x) < PIN


@pytest.mark.parametrize("variant", ["satv", "tvw1", "anat1", "anat2", "apls"])
def test_tv_variants_pinned(variant):
    """The TV gradients of the other TV settings (TVtype 4 and 6, anatomical
    TVtype 1, 2 and 5, APLS) against TVKernel compiled with the variant's
    macro."""
    from oracle import image_oracle as io
    shape = (15, 12, 9)
    rng = np.random.default_rng(51)
    n = int(np.prod(shape))
    u = rng.uniform(0.2, 1.0, n)
    ref = rng.uniform(0.0, 1.0, n)
    # APLS reads the reference image's raw values into sqrt(|d|^2 - (r . d)^2
    # + smooth): reference values below 1 keep it real (above, the reference
    # kernel itself returns NaN)
    S = io.tv_anatomical_tensor(ref, shape, 0.5).astype(np.float64) if variant == "anat1" else \
        (ref if variant == "anat2" else (0.5 * ref if variant == "apls" else None))
    kw = dict(sigma=0.3, C=0.4 if variant == "anat2" else 0.05, S=S)
    ours = io.tv_gradient_variant(u, shape, variant, 1e-3, 0.8, **kw)
    theirs = ref_cl.tv_gradient_variant(u, shape, variant, 1e-3, 0.8, exact_inputs=True, **kw)
    assert orc.rel_l2(ours, theirs) < 1e-12


@pytest.mark.parametrize("l2,diff_type", [(True, 0), (False, 0), (True, 1)])
def test_proxtv_pinned(l2, diff_type):
    """The proximal TV step (image_oracle.proxtv_dual / proxtv_divergence)
    against ProxTVGradient, ProxTVq and ProxTVDivergence compiled with -DPROXTV
    (-DL2 for the L2 ball, -DDIFFTYPE=1 for backward differences), with the
    ball projection active on part of the image."""
    from oracle import image_oracle as io
    shape = (11, 9, 7)
    rng = np.random.default_rng(52)
    n = int(np.prod(shape))
    x = rng.uniform(0.0, 1.0, n)
    q = rng.normal(0.0, 0.3, (3, n))
    rhs = rng.normal(0.0, 1.0, n)
    q_ref, rhs_ref = ref_cl.proxtv_step(x, q, rhs, shape, 0.7, 0.25, l2, diff_type, exact_inputs=True)
    ours = io.proxtv_dual(x, q, shape, 0.7, 0.25, l2, diff_type)
    assert np.abs(ours - q_ref).max() <= 1e-13 * np.abs(q_ref).max()
    r = rhs - io.proxtv_divergence(ours, shape, diff_type)
    assert np.abs(r - rhs_ref).max() <= 1e-13 * np.abs(rhs_ref).max()
    # the projection changed some voxels
    raw = q + 0.7 * np.stack([io._diff(x.reshape(shape, order='F'), a, diff_type == 0).ravel(order='F')
                              for a in range(3)])
    assert np.count_nonzero(np.abs(raw - ours).max(axis=0) > 1e-12) > n // 10


def test_pdhg_proxtv_iteration_pinned():
    """Two PDHG iterations with the proximal TV (oracle.pdhg_tv(prox=...))
    against the same loop built from the reference's kernels: the type-5
    projector pair, ProxTVGradient / ProxTVq / ProxTVDivergence and
    PDHGUpdate."""
    o = _proj("ct_fine5")
    g = orc.Geometry(o)
    R = ref_cl.RefCT(o, exact_inputs=True)
    shape = (g.nx, g.ny, g.nz)
    rng = np.random.default_rng(53)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    y = orc.bdd_forward(g, truth, -1)
    x0 = np.full(g.n_img, 1e-3)
    tau, beta, sigma, sigma2 = 1e-4, 0.01, 1.0, 0.5
    ours = orc.pdhg_tv(g, y, x0, 2, tau, beta, 1e-4, sigma=sigma, prox=dict(sigma2=sigma2, l2=True, diff_type=0))
    x, u = x0.copy(), x0.copy()
    p = np.zeros(g.rays(-1))
    q = np.zeros((3, g.n_img))
    for _ in range(2):
        p = (p + sigma * (R.bdd_forward(x, -1) - y)) / (1.0 + sigma)
        rhs = R.bdd_backward(p, -1)
        q, rhs = ref_cl.proxtv_step(x, q, rhs, shape, sigma2, beta, True, 0, exact_inputs=True)
        x, u = ref_cl.pdhg_update(x, rhs, u, shape, tau, 1.0, 1e-5, exact_inputs=True)
    assert orc.rel_l2(ours, x) < PIN


@pytest.mark.parametrize("l2,three_d", [(True, True), (False, True), (True, False)])
def test_proxtgv_pinned(l2, three_d):
    """One proximal TGV step (image_oracle.proxtgv_step) against
    ProxTVGradient, ProxTVq, ProxTVDivergence, ProxTGVSymmDeriv, ProxTGVq and
    ProxTGVDivergence compiled with -DPROXTV -DPROXTGV (-DTGVZ for 3-D, -DL2
    for the L2 balls), with both ball projections active on part of the
    image."""
    from oracle import image_oracle as io
    shape = (10, 9, 7)
    rng = np.random.default_rng(61)
    n = int(np.prod(shape))
    nr, nv = (6, 3) if three_d else (3, 2)
    x = rng.uniform(0.0, 1.0, n)
    q = rng.normal(0.0, 0.3, (3, n))
    r = rng.normal(0.0, 0.2, (nr, n))
    v = rng.normal(0.0, 0.2, (nv, n))
    rhs = rng.normal(0.0, 1.0, n)
    args = (shape, 0.7, 0.3, 0.2, 0.9, 0.05)
    theirs = ref_cl.proxtgv_step(x, q, r, v, rhs, *args, l2=l2, three_d=three_d, exact_inputs=True)
    ours = io.proxtgv_step(x, q, r, v, rhs, *args, l2=l2, three_d=three_d)
    for a, b in zip(ours, theirs):
        assert np.abs(a - b).max() <= 1e-13 * max(np.abs(b).max(), 1.0)
    # the projections changed part of q and of r
    q_raw = q + 0.7 * (np.stack([io._diff(x.reshape(shape, order='F'), a, True).ravel(order='F') for a in range(3)])
                       - np.vstack([v, np.zeros((3 - nv, n))]))
    assert np.count_nonzero(np.abs(q_raw - ours[0]).max(axis=0) > 1e-12) > n // 10
    rr = ours[1]
    nd = 3 if three_d else 2
    if l2:
        norm = np.sqrt((rr[:nd] ** 2).sum(axis=0) + 2 * (rr[nd:] ** 2).sum(axis=0))
    else:
        norm = np.abs(rr).max(axis=0)
    on_ball = np.abs(norm - 0.2) < 1e-12
    assert n // 10 < np.count_nonzero(on_ball) < n


def test_pdhg_tgv_iteration_pinned():
    """Two PDHG iterations with TGV (oracle.pdhg_tv(tgv=...)) against the same
    loop built from the reference's kernels: the type-5 projector pair, the
    dual step divided by 1 + sigma beta, the six TGV kernels and
    PDHGUpdate."""
    o = _proj("ct_fine5")
    g = orc.Geometry(o)
    R = ref_cl.RefCT(o, exact_inputs=True)
    shape = (g.nx, g.ny, g.nz)
    rng = np.random.default_rng(62)
    truth = rng.uniform(0.0, 0.02, g.n_img)
    y = orc.bdd_forward(g, truth, -1)
    x0 = np.full(g.n_img, 1e-3)
    tau, beta, sigma, sigma2, a0, a1 = 1e-4, 0.5, 1.0, 0.5, 0.01, 0.02
    ours = orc.pdhg_tv(g, y, x0, 2, tau, beta, 1e-4, sigma=sigma,
                       tgv=dict(alpha0=a0, alpha1=a1, sigma2=sigma2, l2=True, three_d=True))
    x, u = x0.copy(), x0.copy()
    p = np.zeros(g.rays(-1))
    q = np.zeros((3, g.n_img))
    r = np.zeros((6, g.n_img))
    v = np.zeros((3, g.n_img))
    for _ in range(2):
        p = (p + sigma * (R.bdd_forward(x, -1) - y)) / (1.0 + sigma * beta)
        rhs = R.bdd_backward(p, -1)
        q, r, v, rhs = ref_cl.proxtgv_step(x, q, r, v, rhs, shape, sigma2, a0, a1, 1.0, tau, True, True,
                                           exact_inputs=True)
        x, u = ref_cl.pdhg_update(x, rhs, u, shape, tau, 1.0, 1e-5, exact_inputs=True)
    assert orc.rel_l2(ours, x) < PIN



@pytest.mark.parametrize("images", [True, False])
def test_rdp_pinned(images):
    """image_oracle.rdp_gradient against RDPKernel compiled with -DRDP: the
    clamp-to-edge texture (USEIMAGES, the reference's built-in default) and
    the buffer path (0 outside), exactly; the two edge rules differ."""
    from oracle import image_oracle as io
    shape = (11, 9, 7)
    rng = np.random.default_rng(71)
    u = rng.uniform(0.0, 2.0, int(np.prod(shape)))
    u[::13] = 0.0
    theirs = ref_cl.rdp_gradient(u, shape, 2.0, 1e-8, 0.3, images=images, exact_inputs=True)
    ours = io.rdp_gradient(u, shape, 2.0, 0.3, 1e-8, clamp=images)
    assert np.abs(ours - theirs).max() <= 1e-14 * np.abs(theirs).max()
    assert orc.rel_l2(io.rdp_gradient(u, shape, 2.0, 0.3, 1e-8, clamp=not images), theirs) > 1e-2


def test_ggmrf_and_hyperbolic_pinned():
    """image_oracle.ggmrf_gradient and hyperbolic_gradient against
    GGMRFKernel (-DGGMRF) and hyperbolicKernel (-DHYPER) compiled on the host
    with a 3 x 3 x 3 window, the image read through the clamp-to-edge texture;
    ties (rounded values) exercise GGMRF's d = 0 skip."""
    from oracle import image_oracle as io
    shape = (9, 8, 7)
    rng = np.random.default_rng(72)
    u = np.round(rng.uniform(0.5, 1.5, int(np.prod(shape))), 2)
    w = rng.uniform(0.2, 1.0, 26)
    p, q, c = 2.0, 1.5, 0.01
    theirs = ref_cl.ggmrf_gradient(u, shape, w, p, q, c, (p - q) / c ** (p - q), 0.3, exact_inputs=True)
    ours = io.ggmrf_gradient(u, shape, (1, 1, 1), w, p, q, c, 0.3)
    assert np.abs(ours - theirs).max() <= 1e-13 * np.abs(theirs).max()
    theirs = ref_cl.hyperbolic_gradient(u, shape, w, 0.7, 0.3, exact_inputs=True)
    ours = io.hyperbolic_gradient(u, shape, (1, 1, 1), w, 0.7, 0.3)
    assert np.abs(ours - theirs).max() <= 1e-13 * np.abs(theirs).max()


@pytest.mark.parametrize("variant,nl_type,extra", [("nlm0", 0, False), ("nlm1", 1, False), ("nlm3", 3, False),
                                                   ("nlm6", 6, False), ("nlm0ar", 0, True)])
def test_nlm_kernel_pinned(variant, nl_type, extra):
    """image_oracle.nlm_gradient in its kernel mode (edges clamped) against
    the reference's NLM kernel compiled on the host: NLM, NLTV, NLRD, NLGGMRF
    and NLM with the adaptive weight and a reference image, search and patch
    windows 3 x 3 x 3."""
    from oracle import image_oracle as io
    shape = (10, 9, 8)
    rng = np.random.default_rng(73)
    n = int(np.prod(shape))
    u = rng.uniform(0.5, 1.5, n)
    gauss = rng.uniform(0.1, 1.0, 27)
    ref = rng.uniform(0.5, 1.5, n) if extra else None
    s = 0.05 if extra else None
    theirs = ref_cl.nlm_gradient(u, shape, gauss, 0.05, 1e-8, 0.3, variant=variant, gamma=2.0,
                                 ggmrf=(2.0, 1.5, 0.01), adaptive_s=s or 0.0, u_ref=ref, exact_inputs=True)
    ours = 0.3 * io.nlm_gradient(u, shape, gauss, (1, 1, 1), (1, 1, 1), 0.05, 1e-8, nl_type, gamma=2.0,
                                 ggmrf=(2.0, 1.5, 0.01), u_ref=ref, adaptive_s=s)
    assert np.count_nonzero(theirs) > n // 2
    assert np.abs(ours - theirs).max() <= 1e-13 * np.abs(theirs).max()


@pytest.mark.parametrize("g", [(2, 3, 1), (1, 1, 1), (3, 2, 2)])
def test_psf_pinned(g):
    """image_oracle.psf_convolve against Convolution3D_f (-DPSF) compiled on
    the host: the window applied at every voxel with the faces mirrored,
    exactly, on an image smaller than some windows' reach in z."""
    from oracle import image_oracle as io
    shape = (13, 11, 9)
    rng = np.random.default_rng(74)
    x = rng.uniform(0.0, 2.0, int(np.prod(shape)))
    w = rng.random((2 * g[0] + 1) * (2 * g[1] + 1) * (2 * g[2] + 1))
    theirs = ref_cl.psf_convolve(x, shape, w, g)
    assert np.abs(io.psf_convolve(x, shape, w, g) - theirs).max() <= 1e-14 * np.abs(theirs).max()


@pytest.mark.parametrize("kind", ["PKMA", "MBSREM", "BSREM"])
@pytest.mark.parametrize("positivity", [True, False])
def test_poisson_update_pinned(kind, positivity):
    """oracle.poisson_update (the image step of the relaxed loops) against
    PoissonUpdate compiled on the host with -DPKMA / -DMBSREM / -DBSREM, with
    values that hit the positivity floor and, for MBSREM, the upper bound."""
    rng = np.random.default_rng(75)
    x = rng.uniform(0.0, 3.0, 500)
    rhs = rng.normal(0.0, 2.0, 500)
    alpha = {"PKMA": 0.7, "MBSREM": 2.5, "BSREM": 0.0}[kind]
    theirs = ref_cl.poisson_update(kind, x, rhs, 0.6, 1e-5, alpha, positivity, exact_inputs=True)
    ours = orc.poisson_update(kind, x, rhs, 0.6, 1e-5, alpha, positivity)
    assert np.abs(ours - theirs).max() <= 1e-15 * np.abs(theirs).max()
    if positivity:
        assert np.any(theirs == 1e-5) or kind == "PKMA"
