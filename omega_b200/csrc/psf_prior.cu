// Image-domain steps around the projectors: the PSF blur and the relative
// difference prior (RDP) gradient.
//
// PSF: Convolution3D_f (auxKernels.cl:192-245) -- a 3-D window of
// (2gx+1)(2gy+1)(2gz+1) weights (x fastest) applied at every voxel, the
// image mirrored at its faces with the edge voxel repeated (index -1 reads 0,
// N reads N-1).  Applied before the forward projection and after the
// backprojection (projfunctions.py:194-200, 1403-1407).
// RDP: RDPKernel (auxKernels.cl:664-872, 6-neighbour form, CUDA border
// addressing: neighbours outside the image read 0):
//   grad += beta * sum_k (u_j - u_k)(gamma |u_j - u_k| + u_j + 3 u_k + eps^2)
//                        / ((u_j + u_k + gamma |u_j - u_k|)^2 + eps)
// with each direction's sum set to 0 when it is NaN.
// Both are stencils over an L2-resident image: one thread per voxel, the
// neighbours served from L1.
#include "kernels.h"

namespace omb {

__device__ __forceinline__ int mirror(int i, int n) {
    if (i < 0) return -i - 1;
    if (i >= n) return n - 1 - (i - n);
    return i;
}

__global__ void k_psf_conv3d(const float *__restrict__ in, float *__restrict__ out, int nx, int ny, int nz,
                             const float *__restrict__ win, int gx, int gy, int gz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int64_t nxy = (int64_t)nx * ny;
    float acc = 0.f;
    int c = 0;
    for (int k = -gz; k <= gz; ++k) {
        const int64_t zo = (int64_t)mirror(z + k, nz) * nxy;
        for (int j = -gy; j <= gy; ++j) {
            const int64_t yo = zo + (int64_t)mirror(y + j, ny) * nx;
            for (int i = -gx; i <= gx; ++i) acc += __ldg(in + yo + mirror(x + i, nx)) * __ldg(win + c++);
        }
    }
    out[x + (int64_t)y * nx + z * nxy] = acc;
}

__device__ __forceinline__ float rdp_term(float uj, float uk, float gamma, float epps) {
    const float d = uj - uk;
    const float div = uj + uk + gamma * fabsf(d);
    return d * (gamma * fabsf(d) + uj + 3.f * uk + epps * epps) / (div * div + epps);
}

__global__ void k_rdp_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz,
                               float gamma, float epps, float beta) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int64_t nxy = (int64_t)nx * ny;
    const int64_t n = x + (int64_t)y * nx + z * nxy;
    const float uj = __ldg(u + n);
    const float xp = x < nx - 1 ? __ldg(u + n + 1) : 0.f, xm = x > 0 ? __ldg(u + n - 1) : 0.f;
    const float yp = y < ny - 1 ? __ldg(u + n + nx) : 0.f, ym = y > 0 ? __ldg(u + n - nx) : 0.f;
    const float zp = z < nz - 1 ? __ldg(u + n + nxy) : 0.f, zm = z > 0 ? __ldg(u + n - nxy) : 0.f;
    // the reference sums the +1 and -1 neighbours as the two halves of a float2
    float a = rdp_term(uj, xp, gamma, epps) + rdp_term(uj, yp, gamma, epps) + rdp_term(uj, zp, gamma, epps);
    float b = rdp_term(uj, xm, gamma, epps) + rdp_term(uj, ym, gamma, epps) + rdp_term(uj, zm, gamma, epps);
    if (isnan(a)) a = 0.f;
    if (isnan(b)) b = 0.f;
    grad[n] += beta * (a + b);
}

}  // namespace omb

using namespace omb;

extern "C" int omb_psf_convolve(const float *in, float *out, int32_t nx, int32_t ny, int32_t nz,
                                const float *window, int32_t gx, int32_t gy, int32_t gz, void *stream) {
    if (!in || !out || !window) return set_error(OMB_ERR_INVALID, "in/out/window pointer is NULL");
    if (in == out) return set_error(OMB_ERR_INVALID, "the PSF convolution cannot run in place");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (gx < 0 || gy < 0 || gz < 0 || gx >= nx || gy >= ny || gz >= nz)
        return set_error(OMB_ERR_INVALID, "window half-widths must be in 0..N-1 (single mirror)");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_psf_conv3d<<<grid, block, 0, (cudaStream_t)stream>>>(in, out, nx, ny, nz, window, gx, gy, gz);
    OMB_LAUNCH_CHECK("PSF convolution launch");
    return OMB_OK;
}

extern "C" int omb_rdp_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float gamma,
                                float epps, float beta, void *stream) {
    if (!u || !grad) return set_error(OMB_ERR_INVALID, "u/grad pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_rdp_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, gamma, epps, beta);
    OMB_LAUNCH_CHECK("RDP gradient launch");
    return OMB_OK;
}
