// Anisotropic-diffusion prior (priors.h:226-237): grad += beta (u - AD(u)) /
// (AD(u) + epps), or beta (u - AD(u)) with no_norm, where AD is ArrayFire's
// anisotropicDiffusion (priors.h:230; ArrayFire is not part of the reference
// tree).  Restated from the published schemes that function implements:
// every slice diffused in 2-D (the third dimension is a batch) with its edges
// replicated, `niter` explicit steps u <- u + dt delta; the conductance
// c(g2) = exp(-g2 / K^2) or 1 / (1 + g2 / K^2) of the squared gradient at the
// half-way point between a voxel and its neighbour (the difference across
// plus a quarter of the squared mean of the two central differences along);
// gradient diffusion (Perona-Malik) delta = sum_axes c_f d_f - c_b d_b, or
// modified curvature diffusion (Whitaker-Xue) with the normalised fluxes
// c d / sqrt(1e-10 + g2), delta = their divergence times the upwind gradient
// magnitude.  One thread per voxel; the 3 x 3 neighbourhood is read through
// the read-only cache; two scratch images (stream-ordered) hold the steps.
#include "common.cuh"
#include "kernels.h"

namespace omb {
namespace {

template <bool MCDE, bool EXPF>
__global__ void __launch_bounds__(256) k_ad_step(const float *__restrict__ in, float *__restrict__ out, int nx, int ny,
                                                 int nz, float dt, float inv_k2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const float *s = in + (int64_t)k * nx * ny;
    const int il = max(i - 1, 0), ir = min(i + 1, nx - 1), jl = max(j - 1, 0), jr = min(j + 1, ny - 1);
    const float C = __ldg(s + i + j * nx), E = __ldg(s + ir + j * nx), W = __ldg(s + il + j * nx);
    const float S = __ldg(s + i + jr * nx), N = __ldg(s + i + jl * nx);
    const float SE = __ldg(s + ir + jr * nx), NE = __ldg(s + ir + jl * nx);
    const float SW = __ldg(s + il + jr * nx), NW = __ldg(s + il + jl * nx);
    const float cx = 0.5f * (E - W), cy = 0.5f * (S - N);
    const float dfx = E - C, dbx = C - W, dfy = S - C, dby = C - N;
    const float tfx = cy + 0.5f * (SE - NE), tbx = cy + 0.5f * (SW - NW);
    const float tfy = cx + 0.5f * (SE - SW), tby = cx + 0.5f * (NE - NW);
    const float gfx = dfx * dfx + 0.25f * tfx * tfx, gbx = dbx * dbx + 0.25f * tbx * tbx;
    const float gfy = dfy * dfy + 0.25f * tfy * tfy, gby = dby * dby + 0.25f * tby * tby;
    auto cond = [&](float g2) { return EXPF ? expf(-g2 * inv_k2) : 1.f / (1.f + g2 * inv_k2); };
    float delta;
    if (!MCDE) {
        delta = cond(gfx) * dfx - cond(gbx) * dbx + cond(gfy) * dfy - cond(gby) * dby;
    } else {
        const float speed = cond(gfx) * dfx / sqrtf(1e-10f + gfx) - cond(gbx) * dbx / sqrtf(1e-10f + gbx) +
                            cond(gfy) * dfy / sqrtf(1e-10f + gfy) - cond(gby) * dby / sqrtf(1e-10f + gby);
        float prop;
        if (speed > 0.f)
            prop = fminf(dbx, 0.f) * fminf(dbx, 0.f) + fmaxf(dfx, 0.f) * fmaxf(dfx, 0.f) +
                   fminf(dby, 0.f) * fminf(dby, 0.f) + fmaxf(dfy, 0.f) * fmaxf(dfy, 0.f);
        else
            prop = fmaxf(dbx, 0.f) * fmaxf(dbx, 0.f) + fminf(dfx, 0.f) * fminf(dfx, 0.f) +
                   fmaxf(dby, 0.f) * fmaxf(dby, 0.f) + fminf(dfy, 0.f) * fminf(dfy, 0.f);
        delta = sqrtf(prop) * speed;
    }
    out[(int64_t)k * nx * ny + i + j * nx] = fmaf(dt, delta, C);
}

__global__ void k_ad_grad(const float *__restrict__ u, const float *__restrict__ a, float *__restrict__ grad,
                          int64_t n, float epps, float beta, int no_norm) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float uu = __ldg(u + i), aa = __ldg(a + i);
        const float g = no_norm ? uu - aa : (uu - aa) / (aa + epps);
        grad[i] += beta * g;
    }
}

}  // namespace
}  // namespace omb

extern "C" int omb_ad_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float dt, float k,
                               int32_t niter, int32_t flux, int32_t diffusion, float epps, float beta, int32_t no_norm,
                               void *stream) {
    using namespace omb;
    if (!u || !grad) return set_error(OMB_ERR_INVALID, "u/grad pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (niter < 1) return set_error(OMB_ERR_INVALID, "AD needs at least one iteration (NiterAD)");
    if (!(k > 0.f)) return set_error(OMB_ERR_INVALID, "AD needs a positive conductance (KAD)");
    if (flux != 1 && flux != 2) return set_error(OMB_ERR_INVALID, "FluxType must be 1 (exponential) or 2 (quadratic)");
    if (diffusion != 1 && diffusion != 2)
        return set_error(OMB_ERR_INVALID, "DiffusionType must be 1 (gradient) or 2 (modified curvature)");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = (int64_t)nx * ny * nz;
    float *buf = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void **>(&buf), 2 * (size_t)n * sizeof(float), st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(OMB_ERR_CUDA, "AD scratch allocation failed");
    }
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    const float inv_k2 = 1.f / (k * k);
    const float *src = u;
    float *dst = buf;
    for (int it = 0; it < niter; ++it) {
        if (diffusion == 2) {
            if (flux == 1) k_ad_step<true, true><<<grid, block, 0, st>>>(src, dst, nx, ny, nz, dt, inv_k2);
            else k_ad_step<true, false><<<grid, block, 0, st>>>(src, dst, nx, ny, nz, dt, inv_k2);
        } else {
            if (flux == 1) k_ad_step<false, true><<<grid, block, 0, st>>>(src, dst, nx, ny, nz, dt, inv_k2);
            else k_ad_step<false, false><<<grid, block, 0, st>>>(src, dst, nx, ny, nz, dt, inv_k2);
        }
        src = dst;
        dst = dst == buf ? buf + n : buf;
    }
    k_ad_grad<<<grid_for(n, 4), kBlock, 0, st>>>(u, src, grad, n, epps, beta, no_norm);
    const cudaError_t le = cudaGetLastError();
    cudaFreeAsync(buf, st);
    if (le != cudaSuccess) return cuda_fail(le, "AD prior launch");
    return OMB_OK;
}
