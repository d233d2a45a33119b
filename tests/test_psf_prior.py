"""PSF blur and the RDP gradient: the projector class's PSF window against
the reference's own PSFKernel (golden fixture psf_pet_mini.npz), the numpy
restatements against direct translations of the reference kernels' index
arithmetic (CPU), and the CUDA kernels against the restatements (GPU)."""
import numpy as np
import pytest

from conftest import load_golden, make_options
from oracle import image_oracle as io
from oracle import oracle as orc


def _psf_options(name="pet_mini"):
    from configs import CONFIGS, apply
    from omega_b200.projector import proj
    o = apply(proj.projectorClass(), dict(CONFIGS[name], use_psf=True, FWHM=np.array([4., 4., 6.])))
    o.addProjector()
    return o


def test_psf_window_matches_reference():
    o = _psf_options()
    p = load_golden("psf", "pet_mini")
    assert [o.g_dim_x, o.g_dim_y, o.g_dim_z] == list(p["g_dim"])
    assert np.array_equal(np.ravel(o.gaussK, order='F'), p["gaussK"])


def _conv_reference_loop(u, shape, w, g):
    """Convolution3D_f's own index arithmetic (auxKernels.cl:199-241), per voxel."""
    nx, ny, nz = shape
    gx, gy, gz = g
    out = np.zeros(nx * ny * nz)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                res, c = 0.0, 0
                for k in range(-gz, gz + 1):
                    if z < gz:
                        zz = abs(k) - 1 - z if k < -z else k + z
                    else:
                        zz = z + k
                        zz = nz - 1 - (zz - nz) if zz >= nz else zz
                    for j in range(-gy, gy + 1):
                        if y < gy:
                            yy = abs(j) - 1 - y if j < -y else j + y
                        else:
                            yy = y + j
                            yy = ny - 1 - (yy - ny) if yy >= ny else yy
                        for i in range(-gx, gx + 1):
                            if x < gx:
                                xx = abs(i) - 1 - x if i < -x else i + x
                            else:
                                xx = x + i
                                xx = nx - 1 - (xx - nx) if xx >= nx else xx
                            res += u[xx + yy * nx + zz * nx * ny] * w[c]
                            c += 1
                out[x + y * nx + z * nx * ny] = res
    return out


def test_psf_restatement_matches_kernel_indexing():
    rng = np.random.default_rng(1)
    shape, g = (7, 5, 6), (2, 1, 2)
    u = rng.random(np.prod(shape))
    w = rng.random((2 * g[0] + 1) * (2 * g[1] + 1) * (2 * g[2] + 1))
    assert np.allclose(io.psf_convolve(u, shape, w, g), _conv_reference_loop(u, shape, w, g), rtol=1e-13)


def _rdp_reference_loop(u, shape, gamma, beta, epps):
    nx, ny, nz = shape
    out = np.zeros(nx * ny * nz)

    def t(uj, uk):
        d = uj - uk
        div = uj + uk + gamma * abs(d)
        return d * (gamma * abs(d) + uj + 3.0 * uk + epps * epps) / (div * div + epps)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                n = x + y * nx + z * nx * ny
                get = (lambda xx, yy, zz: u[xx + yy * nx + zz * nx * ny]
                       if 0 <= xx < nx and 0 <= yy < ny and 0 <= zz < nz else 0.0)
                uj = u[n]
                a = t(uj, get(x + 1, y, z)) + t(uj, get(x, y + 1, z)) + t(uj, get(x, y, z + 1))
                b = t(uj, get(x - 1, y, z)) + t(uj, get(x, y - 1, z)) + t(uj, get(x, y, z - 1))
                out[n] = beta * ((0.0 if np.isnan(a) else a) + (0.0 if np.isnan(b) else b))
    return out


def test_rdp_restatement_matches_kernel():
    rng = np.random.default_rng(2)
    shape = (6, 5, 4)
    u = rng.uniform(0.0, 2.0, np.prod(shape))
    u[3] = 0.0
    got = io.rdp_gradient(u, shape, 2.0, 0.5)
    assert np.allclose(got, _rdp_reference_loop(u, shape, 2.0, 0.5, 1e-8), rtol=1e-12, atol=1e-300)


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


@pytest.mark.gpu
def test_psf_and_rdp_kernels_match_restatements(cuda):
    import ctypes

    import torch
    from omega_b200 import _native, priors
    rng = np.random.default_rng(3)
    shape, g = (37, 29, 19), (2, 3, 1)
    u = rng.uniform(0.0, 2.0, np.prod(shape))
    w = rng.random((2 * g[0] + 1) * (2 * g[1] + 1) * (2 * g[2] + 1))
    w /= w.sum()
    U, W = _t(u, cuda), _t(w, cuda)
    out = torch.empty_like(U)
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    _native.call("omb_psf_convolve", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(out.data_ptr()), *shape,
                 ctypes.c_void_p(W.data_ptr()), *g, st)
    assert orc.rel_l2(out.cpu().numpy(), io.psf_convolve(u, shape, w, g)) < 1e-6
    u[::17] = 0.0
    grad = priors.RDP(_t(u, cuda), *shape, gamma=2.0, beta=0.3).cpu().numpy()
    assert orc.rel_l2(grad, io.rdp_gradient(u, shape, 2.0, 0.3)) < 1e-5
    # the built-in loop's edge rule: neighbours outside the image clamped to the edge voxel
    U2 = _t(u, cuda)
    g2 = torch.zeros_like(U2)
    _native.call("omb_rdp_gradient_ex", ctypes.c_void_p(U2.data_ptr()), ctypes.c_void_p(g2.data_ptr()), *shape, 2.0,
                 1e-8, 0.3, 1, st)
    assert orc.rel_l2(g2.cpu().numpy(), io.rdp_gradient(u, shape, 2.0, 0.3, clamp=True)) < 1e-5
    with pytest.raises(_native.NativeError):
        _native.call("omb_psf_convolve", ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(U.data_ptr()), *shape,
                     ctypes.c_void_p(W.data_ptr()), *g, st)


@pytest.mark.gpu
def test_projections_with_psf(cuda):
    o = _psf_options()
    o.initProj()
    g = orc.Geometry(o)
    shape = (g.nx, g.ny, g.nz)
    gk = np.ravel(o.gaussK, order='F')
    gd = (o.g_dim_x, o.g_dim_y, o.g_dim_z)
    rng = np.random.default_rng(4)
    x = rng.uniform(0.5, 2.0, g.n_img)
    fp = o.forwardProject(_t(x, cuda), 1).cpu().numpy()
    assert orc.rel_l2(fp, orc.forward(g, io.psf_convolve(x, shape, gk, gd), 1)) < 1e-5
    y = rng.uniform(0.0, 2.0, g.rays(1))
    bp, sens = o.backwardProject(_t(y, cuda), 1, sens=True)
    ref_bp, ref_s = orc.backward(g, y, 1, sens=True)
    assert orc.rel_l2(bp.cpu().numpy(), io.psf_convolve(ref_bp, shape, gk, gd)) < 1e-5
    assert orc.rel_l2(sens.cpu().numpy(), io.psf_convolve(ref_s, shape, gk, gd)) < 1e-5


@pytest.mark.parametrize("tag,nd", [("111", (1, 1, 1)), ("221", (2, 2, 1))])
def test_prior_weights_match_reference(tag, nd):
    """computeWeights + quadWeights / huberWeights of the reference
    (golden priorw_pet_mini.npz), and the assembled window's properties."""
    from omega_b200 import priors
    p = load_golden("priorw", "pet_mini")
    o = make_options("pet_mini")
    o.Ndx, o.Ndy, o.Ndz = nd
    w = priors.neighbourhood_weights(o)
    assert np.array_equal(w, p["weights_" + tag])
    wq = priors.normalised_weights(w)
    assert np.array_equal(wq, p["quad_" + tag]) and np.array_equal(wq, p["huber_" + tag])
    win = priors.prior_window(wq, *nd)
    assert abs(float(np.sum(win, dtype=np.float64))) < 1e-6
    shape = (9, 8, 7)
    flat = np.full(np.prod(shape), 3.0)
    assert np.max(np.abs(io.psf_convolve(flat, shape, win, nd))) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("prior", ["Quad", "Huber"])
def test_builtin_osl_quadratic_and_huber(cuda, prior):
    from omega_b200 import priors
    from omega_b200 import reconstruction as rec
    o = make_options("pet_mini")
    g = orc.Geometry(o)
    rng = np.random.default_rng(5)
    truth = rng.uniform(0.5, 2.0, g.n_img)
    full = make_options("pet_mini")
    full.subsets, full.subsetType = 1, 8
    full.addProjector()
    y = rng.poisson(orc.forward(orc.Geometry(full), truth, 0) * 200).astype(np.float32) / 200
    o.SinM = y.copy()
    o.OSL_OSEM = True
    setattr(o, prior, True)
    o.beta = 0.002  # one-step-late stays well-conditioned at this weight (see the RDP case)
    o.huber_delta = 0.05
    o.Niter = 2
    out, _ = rec.reconstructions_main(o)
    m = np.asarray(o.SinM, dtype=np.float32).ravel(order='F')
    ys = [np.asarray(o.subsetMeasurements(m, s), dtype=np.float64) for s in range(g.n_subsets)]
    shape = (g.nx, g.ny, g.nz)
    win = priors.prior_window(priors.normalised_weights(priors.neighbourhood_weights(o)), 1, 1, 1)
    delta = 0.05 if prior == "Huber" else np.inf

    def grad(x):
        return 0.002 * np.clip(io.psf_convolve(x, shape, win, (1, 1, 1)), -delta, delta)
    ref = orc.osem(g, ys, np.ones(g.n_img), 2, prior_grad=grad)
    assert orc.rel_l2(out.ravel(order='F'), ref) < 5e-5, orc.rel_l2(out.ravel(order='F'), ref)
    assert orc.rel_l2(ref, orc.osem(g, ys, np.ones(g.n_img), 2)) > 1e-4
