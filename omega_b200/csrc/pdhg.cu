// PDHG with a TV-gradient term (one subset) and the power method that sets
// its primal step.
//
// dual:    p = (p + sigma * (A x - y)) / (1 + sigma)      computeForwardProject.h:227-316
// primal:  rhs = A^T p + beta * grad TV(x)                priors.h:404-409 -> auxKernels.cl:1733
//          u' = max(epps, u - tau * rhs);  x = u' + theta (u' - u)   auxKernels.cl:2034-2062 (PDHGUpdate)
// TV:      smoothed isotropic TV gradient of TVKernel (auxKernels.cl:1733-1990, plain TV, no
//          reference image); neighbours outside the volume read the edge voxel, as the
//          reference's point-sampled clamp-to-edge texture does (ProjectorClass.h:6541-6580).
// power method: L = max eig(A^T A), tau = 1/L (functions.hpp:2417-2540, 2886-2905).
#include "kernels.h"

namespace omb {

__global__ void k_pdhg_dual(float *__restrict__ p, const float *__restrict__ fp, const float *__restrict__ y,
                            int64_t n, float sigma) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const float inv = 1.f / (1.f + sigma);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        p[i] = (p[i] + sigma * (__ldg(fp + i) - __ldg(y + i))) * inv;
}

__device__ __forceinline__ float tv_at(const float *__restrict__ u, int x, int y, int z, int nx, int ny, int nz) {
    x = min(max(x, 0), nx - 1);
    y = min(max(y, 0), ny - 1);
    z = min(max(z, 0), nz - 1);
    return __ldg(u + x + (int64_t)y * nx + (int64_t)z * nx * ny);
}

// Smoothed isotropic TV gradient at voxel (i, j, k) (TVKernel, plain TV).
__device__ __forceinline__ float tv_grad(const float *__restrict__ x, int i, int j, int k, int nx, int ny, int nz,
                                         float smooth) {
    const float c = tv_at(x, i, j, k, nx, ny, nz);
    const float px = tv_at(x, i + 1, j, k, nx, ny, nz), py = tv_at(x, i, j + 1, k, nx, ny, nz),
                pz = tv_at(x, i, j, k + 1, nx, ny, nz);
    const float mx = tv_at(x, i - 1, j, k, nx, ny, nz), my = tv_at(x, i, j - 1, k, nx, ny, nz),
                mz = tv_at(x, i, j, k - 1, nx, ny, nz);
    const float uix = tv_at(x, i - 1, j + 1, k, nx, ny, nz), uiy = tv_at(x, i - 1, j, k + 1, nx, ny, nz);
    const float ujx = tv_at(x, i + 1, j - 1, k, nx, ny, nz), ujy = tv_at(x, i, j - 1, k + 1, nx, ny, nz);
    const float ukx = tv_at(x, i + 1, j, k - 1, nx, ny, nz), uky = tv_at(x, i, j + 1, k - 1, nx, ny, nz);
    const float a0 = px - c, a1 = py - c, a2 = pz - c;
    const float p0 = sqrtf(a0 * a0 + a1 * a1 + a2 * a2 + smooth);
    const float b0 = c - mx, b1 = uix - mx, b2 = uiy - mx;
    const float p1 = sqrtf(b0 * b0 + b1 * b1 + b2 * b2 + smooth);
    const float c0 = ujx - my, c1 = c - my, c2 = ujy - my;
    const float p2 = sqrtf(c0 * c0 + c1 * c1 + c2 * c2 + smooth);
    const float d0 = ukx - mz, d1 = uky - mz, d2 = c - mz;
    const float p3 = sqrtf(d0 * d0 + d1 * d1 + d2 * d2 + smooth);
    return (3.f * c - px - py - pz) / p0 + (c - mx) / p1 + (c - my) / p2 + (c - mz) / p3 + 1e-7f;
}

// grad += beta * the TV gradient (the TV prior of the one-step-late and
// relaxed algorithms, priors.h:404-409).
__global__ void __launch_bounds__(256) k_tv_gradient(const float *__restrict__ x, float *__restrict__ grad, int nx,
                                                     int ny, int nz, float beta, float smooth) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    grad[i + (int64_t)j * nx + (int64_t)k * nx * ny] += beta * tv_grad(x, i, j, k, nx, ny, nz, smooth);
}

// Primal step fused with the TV gradient: reads x (stencil), rhs and u,
// writes u and the extrapolated image into x_out (x_out != x).
__global__ void __launch_bounds__(256) k_pdhg_primal_tv(const float *__restrict__ x, const float *__restrict__ rhs,
                                                        float *__restrict__ u, float *__restrict__ x_out, int nx,
                                                        int ny, int nz, float beta, float smooth, float tau,
                                                        float theta, float epps, int positivity) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t n = i + (int64_t)j * nx + (int64_t)k * nx * ny;
    const float g = beta != 0.f ? beta * tv_grad(x, i, j, k, nx, ny, nz, smooth) : 0.f;
    const float r = __ldg(rhs + n) + g;
    const float uprev = u[n];
    float unew = uprev - tau * r;
    if (positivity) unew = fmaxf(epps, unew);
    u[n] = unew;
    x_out[n] = unew + theta * (unew - uprev);
}

// FP64 dot products a.b (and b.b) with a deterministic two-pass reduction.
constexpr int kDotBlocks = 592;

__global__ void __launch_bounds__(256) k_dot2(const float *__restrict__ a, const float *__restrict__ b, int64_t n,
                                              double *__restrict__ part) {
    __shared__ double sh[2][8];
    double ab = 0.0, bb = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = __ldg(a + i), y = __ldg(b + i);
        ab += x * y;
        bb += y * y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        ab += __shfl_down_sync(0xffffffffu, ab, o);
        bb += __shfl_down_sync(0xffffffffu, bb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = ab;
        sh[1][threadIdx.x >> 5] = bb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < 8; ++w) {
            s0 += sh[0][w];
            s1 += sh[1][w];
        }
        part[2 * blockIdx.x] = s0;
        part[2 * blockIdx.x + 1] = s1;
    }
}

__global__ void k_dot2_fold(const double *__restrict__ part, int nb, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int i = 0; i < nb; ++i) {
            s0 += part[2 * i];
            s1 += part[2 * i + 1];
        }
        out[0] = s0;
        out[1] = s1;
    }
}

// x = b / sqrt(bb) with bb read on the device (no host round trip).
__global__ void k_normalize_into(float *__restrict__ x, const float *__restrict__ b, int64_t n,
                                 const double *__restrict__ dots) {
    const float inv = (float)(1.0 / sqrt(dots[1]));
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = __ldg(b + i) * inv;
}

int pdhg_dual(float *p, const float *fp, const float *y, int64_t n, float sigma, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_pdhg_dual<<<grid_for(n, 4), kBlock, 0, st>>>(p, fp, y, n, sigma);
    OMB_LAUNCH_CHECK("pdhg dual launch");
    return OMB_OK;
}

int pdhg_primal_tv(const Grid &g, const float *x, const float *rhs, float *u, float *x_out, float beta, float smooth,
                   float tau, float theta, float epps, int positivity, cudaStream_t st) {
    if (g.nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    dim3 block(32, 8);
    dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
    k_pdhg_primal_tv<<<grid, block, 0, st>>>(x, rhs, u, x_out, g.nx, g.ny, g.nz, beta, smooth, tau, theta, epps,
                                             positivity);
    OMB_LAUNCH_CHECK("pdhg primal launch");
    return OMB_OK;
}

size_t dot_workspace_bytes() { return (size_t)(2 * kDotBlocks + 2) * sizeof(double); }

// dots[0] = a.b, dots[1] = b.b (device doubles at work + 2*kDotBlocks).
int dot2(const float *a, const float *b, int64_t n, double *work, cudaStream_t st) {
    k_dot2<<<kDotBlocks, 256, 0, st>>>(a, b, n, work);
    OMB_LAUNCH_CHECK("dot launch");
    k_dot2_fold<<<1, 32, 0, st>>>(work, kDotBlocks, work + 2 * kDotBlocks);
    OMB_LAUNCH_CHECK("dot fold launch");
    return OMB_OK;
}

int normalize_into(float *x, const float *b, int64_t n, const double *dots, cudaStream_t st) {
    k_normalize_into<<<grid_for(n, 4), kBlock, 0, st>>>(x, b, n, dots);
    OMB_LAUNCH_CHECK("normalize launch");
    return OMB_OK;
}

}  // namespace omb

extern "C" int omb_tv_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float beta,
                               float smooth, void *stream) {
    using namespace omb;
    if (!u || !grad) return set_error(OMB_ERR_INVALID, "u/grad pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_tv_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, beta, smooth);
    OMB_LAUNCH_CHECK("TV gradient launch");
    return OMB_OK;
}
