"""TEST INFRASTRUCTURE ONLY -- FP64 numpy restatements of the image-domain
steps around the projectors, for the parity tests:

* psf_convolve: Convolution3D_f (OMEGA source/opencl/auxKernels.cl:192-245),
  the window applied at every voxel with the image mirrored at its faces
  (edge voxel repeated: index -1 reads 0, N reads N-1);
* rdp_gradient: RDPKernel (auxKernels.cl:664-872), 6-neighbour form,
  neighbours outside the image 0 (the CUDA border addressing of the
  reference's PyTorch/CuPy path, util/priors.py:178-181).
"""
import numpy as np


def psf_convolve(img, shape, window, g):
    """img: flat, x fastest; window: flat (2gx+1)(2gy+1)(2gz+1), x fastest."""
    nx, ny, nz = shape
    gx, gy, gz = (int(v) for v in g)
    u = np.asarray(img, dtype=np.float64).reshape((nx, ny, nz), order='F')
    w = np.asarray(window, dtype=np.float64).reshape((2 * gx + 1, 2 * gy + 1, 2 * gz + 1), order='F')
    p = np.pad(u, ((gx, gx), (gy, gy), (gz, gz)), mode='symmetric')
    out = np.zeros_like(u)
    for k in range(2 * gz + 1):
        for j in range(2 * gy + 1):
            for i in range(2 * gx + 1):
                out += w[i, j, k] * p[i:i + nx, j:j + ny, k:k + nz]
    return out.ravel(order='F')


def rdp_gradient(u, shape, gamma, beta, epps=1e-8):
    nx, ny, nz = shape
    a = np.asarray(u, dtype=np.float64).reshape((nx, ny, nz), order='F')
    p = np.pad(a, 1, mode='constant')

    def term(k):
        d = a - k
        div = a + k + gamma * np.abs(d)
        return d * (gamma * np.abs(d) + a + 3.0 * k + epps * epps) / (div * div + epps)

    c = p[1:-1, 1:-1, 1:-1]
    plus = term(p[2:, 1:-1, 1:-1]) + term(p[1:-1, 2:, 1:-1]) + term(p[1:-1, 1:-1, 2:])
    minus = term(p[:-2, 1:-1, 1:-1]) + term(p[1:-1, :-2, 1:-1]) + term(p[1:-1, 1:-1, :-2])
    plus[np.isnan(plus)] = 0.0
    minus[np.isnan(minus)] = 0.0
    assert c.shape == a.shape
    return (beta * (plus + minus)).ravel(order='F')
