// Image-domain steps around the projectors: the PSF blur, the relative
// difference prior (RDP) gradient and the non-local (NLM family) gradients.
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

// CLAMP: a neighbour outside the image reads the edge voxel (the clamp-to-edge
// texture of the reference's built-in path with useImages, ProjectorClass.h:
// 6574-6576; samplerRDP auxKernels.cl:653), else 0 (its buffer path, and the
// border-addressed texture of util/priors.py:143-146)
template <bool CLAMP>
__global__ void k_rdp_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz,
                               float gamma, float epps, float beta) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int64_t nxy = (int64_t)nx * ny;
    const int64_t n = x + (int64_t)y * nx + z * nxy;
    const float uj = __ldg(u + n);
    const float e = CLAMP ? uj : 0.f;
    const float xp = x < nx - 1 ? __ldg(u + n + 1) : e, xm = x > 0 ? __ldg(u + n - 1) : e;
    const float yp = y < ny - 1 ? __ldg(u + n + nx) : e, ym = y > 0 ? __ldg(u + n - nx) : e;
    const float zp = z < nz - 1 ? __ldg(u + n + nxy) : e, zm = z > 0 ? __ldg(u + n - nxy) : e;
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
    k_rdp_gradient<false><<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, gamma, epps, beta);
    OMB_LAUNCH_CHECK("RDP gradient launch");
    return OMB_OK;
}

extern "C" int omb_rdp_gradient_ex(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float gamma,
                                   float epps, float beta, int32_t edge, void *stream) {
    if (edge != 0 && edge != 1) return set_error(OMB_ERR_INVALID, "edge must be 0 (zero) or 1 (clamp)");
    if (!u || !grad) return set_error(OMB_ERR_INVALID, "u/grad pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    if (edge) k_rdp_gradient<true><<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, gamma, epps, beta);
    else k_rdp_gradient<false><<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, gamma, epps, beta);
    OMB_LAUNCH_CHECK("RDP gradient launch");
    return OMB_OK;
}

namespace omb {

// Non-local regularisers (the NLM kernel, auxKernels.cl:297-620, with the
// image read clamped to its edges as the reference's texture sampler reads
// it): for voxel j, over the search offsets k != 0 with patch distance
// d_k = sum_p g_p (P(j + p) - P(j + k + p))^2 (P the reference image when one
// is given) and weight w_k = exp(-d_k / h), W = epps + sum_k w_k:
//   0 NLM      sum w (u_j - u_k) / W
//   1 NLTV     the same / sqrt((epps + sum w (u_j - u_k)^2) / W + epps)
//   2 NLM-MRP  u_j - sum w u_k / W
//   3 NLRD     sum w d (gamma |d| + u_j + 3 u_k + epps^2) / (u_j + u_k + gamma |d| + epps)^2 / W
//   4 NL Lange sum w (s - s / (|d| / gamma + 1)) / W, s = sign(d)
//   5 NLM-MRP with Lange applied to it
//   6 NLGGMRF  sum w |d|^(p-1) / (1 + |d / c|^(p-q)) (p - gamma |d|^(p-q) / (1 + |d/c|^(p-q))) s / W
// (d = u_j - u_k) and grad += beta * that; with `adaptive` (NLMADAPTIVE)
// w_k = exp(-d_k / (d_k / |patch| * h + s)).  One thread per voxel; the image
// is L2-resident and its neighbourhood served from L1.
__device__ __forceinline__ int clampi(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
__device__ __forceinline__ float sgnn(float v) { return (float)((0.f < v) - (v < 0.f)); }

template <int TYPE>
__global__ void k_nlm(const float *__restrict__ u, const float *__restrict__ ref, float *__restrict__ grad, int nx,
                      int ny, int nz, int sx, int sy, int sz, int px, int py, int pz, const float *__restrict__ gauss,
                      float h, float epps, float beta, float gamma, float gp, float gq, float gc, int adaptive,
                      float adapt_s) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int64_t nxy = (int64_t)nx * ny;
    const float *P = ref ? ref : u;
    auto at = [&](const float *a, int xx, int yy, int zz) {
        return __ldg(a + clampi(xx, nx) + (int64_t)clampi(yy, ny) * nx + (int64_t)clampi(zz, nz) * nxy);
    };
    const float uj = __ldg(u + x + (int64_t)y * nx + (int64_t)z * nxy);
    float wsum = epps, out = 0.f, ala = epps;
    const float cpq = TYPE == 6 ? powf(gc, gp - gq) : 0.f;
    const float psize = (float)((2 * px + 1) * (2 * py + 1) * (2 * pz + 1));
    for (int i = -sx; i <= sx; ++i)
        for (int j = -sy; j <= sy; ++j)
            for (int k = -sz; k <= sz; ++k) {
                if (i == 0 && j == 0 && k == 0) continue;
                float dist = 0.f;
                for (int qz = -pz; qz <= pz; ++qz)
                    for (int qy = -py; qy <= py; ++qy) {
                        int dg = (qz + pz) * (2 * px + 1) * (2 * py + 1) + (qy + py) * (2 * px + 1);
                        for (int qx = -px; qx <= px; ++qx) {
                            const float gg = __ldg(gauss + dg++);
                            const float d = at(P, x + qx, y + qy, z + qz) - at(P, x + i + qx, y + j + qy, z + k + qz);
                            dist += gg * d * d;
                        }
                    }
                // NLMADAPTIVE: h scaled by the patch's mean squared difference plus a constant
                const float w = adaptive ? expf(-dist / ((dist / psize) * h + adapt_s)) : expf(-dist / h);
                wsum += w;
                const float uk = at(u, x + i, y + j, z + k);
                if (TYPE == 2 || TYPE == 5) {
                    out += w * uk;
                } else if (TYPE == 0) {
                    out += w * (uj - uk);
                } else if (TYPE == 3) {
                    const float d = uj - uk;
                    const float dp = uj + uk + gamma * fabsf(d) + epps;
                    out += w * d * (gamma * fabsf(d) + uj + 3.f * uk + epps * epps) / (dp * dp);
                } else if (TYPE == 4) {
                    const float d = uj - uk;
                    const float s = sgnn(d);
                    out += w * (s - s / (fabsf(d) / gamma + 1.f));
                } else if (TYPE == 6) {
                    const float d = uj - uk;
                    const float dcpq = powf(fabsf(d / gc), gp - gq);
                    const float dpq = 1.f + dcpq;
                    out += w * (powf(fabsf(d), gp - 1.f) / dpq) * (gp - gamma * ((dcpq * cpq) / dpq)) * sgnn(d);
                } else {
                    const float d = uj - uk;
                    out += w * d;
                    ala += w * d * d;
                }
            }
    wsum = 1.f / wsum;
    out *= wsum;
    if (TYPE == 2) {
        out = uj - out;
    } else if (TYPE == 5) {
        out = uj - out;
        const float s = sgnn(out);
        out = s - s / (fabsf(out) / gamma + 1.f);
    } else if (TYPE == 1) {
        out /= sqrtf(ala * wsum + epps);
    }
    grad[x + (int64_t)y * nx + (int64_t)z * nxy] += beta * out;
}

}  // namespace omb

extern "C" int omb_nlm_gradient(const float *u, const float *ref, float *grad, int32_t nx, int32_t ny, int32_t nz,
                                const int32_t *search, const int32_t *patch, const float *gaussian, float h,
                                float epps, float beta, int32_t type, float gamma, const float *ggmrf_pqc,
                                int32_t adaptive, float adaptive_s, void *stream) {
    using namespace omb;
    if (!u || !grad || !gaussian || !search || !patch) return set_error(OMB_ERR_INVALID, "NULL pointer passed to omb_nlm_gradient");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    for (int a = 0; a < 3; ++a)
        if (search[a] < 0 || search[a] > 16 || patch[a] < 0 || patch[a] > 16)
            return set_error(OMB_ERR_INVALID, "NLM windows must be in 0..16");
    if (!(h > 0.f)) return set_error(OMB_ERR_INVALID, "NLM filter parameter h must be positive");
    if (type == 6 && !ggmrf_pqc) return set_error(OMB_ERR_INVALID, "NLGGMRF needs p, q and c");
    const float gp = type == 6 ? ggmrf_pqc[0] : 0.f, gq = type == 6 ? ggmrf_pqc[1] : 0.f,
                gc = type == 6 ? ggmrf_pqc[2] : 1.f;
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    cudaStream_t st = (cudaStream_t)stream;
#define OMB_NLM(T)                                                                                                \
    k_nlm<T><<<grid, block, 0, st>>>(u, ref, grad, nx, ny, nz, search[0], search[1], search[2], patch[0], patch[1], \
                                     patch[2], gaussian, h, epps, beta, gamma, gp, gq, gc, \
                                     adaptive != 0, adaptive_s)
    switch (type) {
        case 0: OMB_NLM(0); break;
        case 1: OMB_NLM(1); break;
        case 2: OMB_NLM(2); break;
        case 3: OMB_NLM(3); break;
        case 4: OMB_NLM(4); break;
        case 5: OMB_NLM(5); break;
        case 6: OMB_NLM(6); break;
        default: return set_error(OMB_ERR_INVALID, "NLM type must be 0..6");
    }
#undef OMB_NLM
    OMB_LAUNCH_CHECK("NLM gradient launch");
    return OMB_OK;
}

namespace omb {

// Median root prior (MRP, priors.h:4-25 with medianFilter3D,
// auxKernels.cl:981-1027): the median of the (2mx+1)(2my+1)(2mz+1)
// neighbourhood of the image mirrored at its faces (padding(),
// functions.hpp:216-260: index -1 reads 0), the element of rank K / 2 with
// ties ranked by position; grad += beta * (u - med) / (med + epps), or
// beta * (u - med) with no_norm.  One thread per voxel, the window in local
// memory (K <= 125).
constexpr int kMrpMax = 125;

__global__ void k_mrp_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz, int mx,
                               int my, int mz, float epps, float beta, int no_norm) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int64_t nxy = (int64_t)nx * ny;
    float win[kMrpMax];
    int k = 0;
    for (int i = -mx; i <= mx; ++i)
        for (int j = -my; j <= my; ++j)
            for (int l = -mz; l <= mz; ++l)
                win[k++] = __ldg(u + mirror(x + i, nx) + (int64_t)mirror(y + j, ny) * nx + (int64_t)mirror(z + l, nz) * nxy);
    float med = win[0];
    for (int h = 0; h < k; ++h) {
        int rank = 0;
        for (int l = 0; l < k; ++l) rank += (win[h] > win[l] || (win[h] == win[l] && h < l)) ? 1 : 0;
        if (rank == k / 2) {
            med = win[h];
            break;
        }
    }
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nxy;
    const float d = __ldg(u + n) - med;
    grad[n] += no_norm ? d * beta : d / (med + epps) * beta;
}

}  // namespace omb

extern "C" int omb_mrp_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx,
                                int32_t my, int32_t mz, float epps, float beta, int32_t no_norm, void *stream) {
    using namespace omb;
    if (!u || !grad) return set_error(OMB_ERR_INVALID, "u/grad pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (mx < 0 || my < 0 || mz < 0 || (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1) > kMrpMax)
        return set_error(OMB_ERR_UNSUPPORTED, "MRP windows of more than 125 voxels are not built");
    if (mx > nx || my > ny || mz > nz) return set_error(OMB_ERR_INVALID, "MRP window larger than the image");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_mrp_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, mx, my, mz, epps, beta, no_norm);
    OMB_LAUNCH_CHECK("MRP gradient launch");
    return OMB_OK;
}

namespace omb {

// GGMRF prior (GGMRFKernel, auxKernels.cl:878-980; the image read clamped to
// its edges): grad += beta * sum_k w_k |d|^(p-1) / (1 + |d / c|^(p-q))
//   * (p - pqc |d / c|^(p-q) c^(p-q) / (1 + |d / c|^(p-q))) * sign(d),
// d = u_j - u_k over the neighbours (x outermost, z fastest, centre skipped),
// pqc = (p - q) / c^(p-q) (libHeader.h:1180), terms with d = 0 left out.
__global__ void k_ggmrf_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz, int sx,
                                 int sy, int sz, const float *__restrict__ w, float p, float q, float c, float pqc,
                                 float beta) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int64_t nxy = (int64_t)nx * ny;
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nxy;
    const float uj = __ldg(u + n);
    const float cpq = powf(c, p - q);
    float out = 0.f;
    int uu = 0;
    for (int i = -sx; i <= sx; ++i)
        for (int j = -sy; j <= sy; ++j)
            for (int k = -sz; k <= sz; ++k) {
                if (i == 0 && j == 0 && k == 0) continue;
                const float uk =
                    __ldg(u + clampi(x + i, nx) + (int64_t)clampi(y + j, ny) * nx + (int64_t)clampi(z + k, nz) * nxy);
                const float d = uj - uk;
                if (d != 0.f) {
                    const float dcpq = powf(fabsf(d / c), p - q);
                    const float dpq = 1.f + dcpq;
                    out += __ldg(w + uu) * (powf(fabsf(d), p - 1.f) / dpq) * (p - pqc * ((dcpq * cpq) / dpq)) * sgnn(d);
                }
                ++uu;
            }
    grad[n] += beta * out;
}

}  // namespace omb

extern "C" int omb_ggmrf_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t sx,
                                  int32_t sy, int32_t sz, const float *weights, float p, float q, float c, float beta,
                                  void *stream) {
    using namespace omb;
    if (!u || !grad || !weights) return set_error(OMB_ERR_INVALID, "u/grad/weights pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (sx < 0 || sy < 0 || sz < 0 || sx > 8 || sy > 8 || sz > 8) return set_error(OMB_ERR_INVALID, "GGMRF window 0..8");
    if (!(c > 0.f)) return set_error(OMB_ERR_INVALID, "GGMRF needs c > 0");
    const float pqc = (p - q) / powf(c, p - q);
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_ggmrf_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, sx, sy, sz, weights, p, q, c, pqc,
                                                                beta);
    OMB_LAUNCH_CHECK("GGMRF gradient launch");
    return OMB_OK;
}

namespace omb {

// Hyperbolic prior (hyperbolicKernel, auxKernels.cl:1591-1688; the image read
// clamped to its edges): grad += beta * sum_k w_k t_k / delta / sqrt(t_k^2 + 1),
// t_k = (u_j - u_k) / delta, over the neighbours z outermost, x fastest.
__global__ void k_hyperbolic_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz,
                                      int sx, int sy, int sz, const float *__restrict__ w, float delta, float beta) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int64_t nxy = (int64_t)nx * ny;
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nxy;
    const float uj = __ldg(u + n);
    const float inv = 1.f / delta;
    float out = 0.f;
    int uu = 0;
    for (int k = -sz; k <= sz; ++k)
        for (int j = -sy; j <= sy; ++j)
            for (int i = -sx; i <= sx; ++i) {
                if (i == 0 && j == 0 && k == 0) continue;
                const float uk =
                    __ldg(u + clampi(x + i, nx) + (int64_t)clampi(y + j, ny) * nx + (int64_t)clampi(z + k, nz) * nxy);
                const float t = (uj - uk) * inv;
                out += t * inv * rsqrtf(t * t + 1.f) * __ldg(w + uu++);
            }
    grad[n] += beta * out;
}

}  // namespace omb

extern "C" int omb_hyperbolic_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t sx,
                                       int32_t sy, int32_t sz, const float *weights, float delta, float beta,
                                       void *stream) {
    using namespace omb;
    if (!u || !grad || !weights) return set_error(OMB_ERR_INVALID, "u/grad/weights pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (sx < 0 || sy < 0 || sz < 0 || sx > 8 || sy > 8 || sz > 8)
        return set_error(OMB_ERR_INVALID, "hyperbolic prior window 0..8");
    if (!(delta > 0.f)) return set_error(OMB_ERR_INVALID, "the hyperbolic prior needs delta > 0");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_hyperbolic_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, sx, sy, sz, weights, delta,
                                                                     beta);
    OMB_LAUNCH_CHECK("hyperbolic gradient launch");
    return OMB_OK;
}

namespace omb {

// Weighted-mean prior, mean types 1-3 (Weighted_mean, priors.h:99-160 for
// types 1-3): m = the weighted arithmetic (1), harmonic (2) or geometric (3)
// mean of the (2mx+1)(2my+1)(2mz+1) window of u mirrored at its faces, the
// weights w (x fastest) applied as a convolution (af::convolve3: the weight
// of offset -o multiplies u(x + o)) and divided by wsum;
// grad += beta * (u - m) / (m + epps), or beta * (u - m) with no_norm.
__global__ void k_wmean_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz, int mx,
                                 int my, int mz, const float *__restrict__ w, float wsum, int mean_type, float epps,
                                 float beta, int no_norm) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int64_t nxy = (int64_t)nx * ny;
    const int wx = 2 * mx + 1, wy = 2 * my + 1;
    float acc = 0.f;
    for (int k = -mz; k <= mz; ++k)
        for (int j = -my; j <= my; ++j)
            for (int i = -mx; i <= mx; ++i) {
                const float v = __ldg(u + mirror(x + i, nx) + (int64_t)mirror(y + j, ny) * nx +
                                      (int64_t)mirror(z + k, nz) * nxy);
                const float wk = __ldg(w + (mx - i) + (my - j) * wx + (mz - k) * wx * wy) / wsum;
                acc += wk * (mean_type == 2 ? 1.f / v : (mean_type == 3 ? logf(v) : v));
            }
    const float m = mean_type == 2 ? 1.f / acc : (mean_type == 3 ? expf(acc) : acc);
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nxy;
    const float d = __ldg(u + n) - m;
    grad[n] += beta * (no_norm ? d : d / (m + epps));
}

// Mean types 4-6, first pass: the weighted mean M over the image grown by
// (mx, my, mz) on every side (the means of the neighbours of border voxels),
// from the image mirrored twice as far; M(c) for c = the original
// coordinate, stored at c + (mx, my, mz) in an (nx+2mx)(ny+2my)(nz+2mz) grid.
__global__ void k_wmean_ext(const float *__restrict__ u, float *__restrict__ mext, int nx, int ny, int nz, int mx,
                            int my, int mz, const float *__restrict__ w, float wsum, int mean_type) {
    const int ex = nx + 2 * mx, ey = ny + 2 * my;
    const int xe = blockIdx.x * blockDim.x + threadIdx.x;
    const int ye = blockIdx.y * blockDim.y + threadIdx.y;
    const int ze = blockIdx.z;
    if (xe >= ex || ye >= ey) return;
    const int x = xe - mx, y = ye - my, z = ze - mz;
    const int64_t nxy = (int64_t)nx * ny;
    const int wx = 2 * mx + 1, wy = 2 * my + 1;
    float acc = 0.f;
    for (int k = -mz; k <= mz; ++k)
        for (int j = -my; j <= my; ++j)
            for (int i = -mx; i <= mx; ++i) {
                const float v = __ldg(u + mirror(x + i, nx) + (int64_t)mirror(y + j, ny) * nx +
                                      (int64_t)mirror(z + k, nz) * nxy);
                const float wk = __ldg(w + (mx - i) + (my - j) * wx + (mz - k) * wx * wy) / wsum;
                acc += wk * (mean_type == 5 ? 1.f / v : (mean_type == 6 ? logf(v) : v));
            }
    mext[xe + (int64_t)ye * ex + (int64_t)ze * ex * ey] =
        mean_type == 5 ? 1.f / acc : (mean_type == 6 ? expf(acc) : acc);
}

// Second pass (priors.h:125-210): per voxel the sum over the window's
// offsets d of w_d g(u, M(x + d)), the raw weights paired with the offsets
// in x-fastest order: type 4 log(max(u / M, 1e-6)); type 5, with u' =
// max(u, 1e-6), (u' - M) / u' - ((u' - M) / (sqrt(2) u'))^2; type 6
// 1 - M / u'.
__global__ void k_wmean_grad46(const float *__restrict__ u, const float *__restrict__ mext, float *__restrict__ grad,
                               int nx, int ny, int nz, int mx, int my, int mz, const float *__restrict__ w,
                               int mean_type, float beta) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int ex = nx + 2 * mx, ey = ny + 2 * my;
    const int wx = 2 * mx + 1, wy = 2 * my + 1;
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nx * ny;
    const float uv = __ldg(u + n);
    const float ut = fmaxf(uv, 1e-6f);
    const float s2 = sqrtf(2.f) * ut;
    float acc = 0.f;
    for (int l = 0; l < 2 * mz + 1; ++l)
        for (int k = 0; k < wy; ++k)
            for (int h = 0; h < wx; ++h) {
                // offset (h - mx, k - my, l - mz): extended index (x + h, y + k, z + l)
                const float M = __ldg(mext + (x + h) + (int64_t)(y + k) * ex + (int64_t)(z + l) * ex * ey);
                const float wk = __ldg(w + h + k * wx + l * wx * wy);
                float g;
                if (mean_type == 4) {
                    g = logf(fmaxf(uv / M, 1e-6f));
                } else if (mean_type == 5) {
                    const float d = ut - M;
                    const float r = d / s2;
                    g = d / ut - r * r;
                } else {
                    g = 1.f - M / ut;
                }
                acc += g * wk;
            }
    grad[n] += beta * acc;
}

}  // namespace omb

extern "C" int omb_wmean_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx,
                                  int32_t my, int32_t mz, const float *weights, float wsum, int32_t mean_type,
                                  float epps, float beta, int32_t no_norm, void *stream) {
    using namespace omb;
    if (!u || !grad || !weights) return set_error(OMB_ERR_INVALID, "u/grad/weights pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (mean_type < 1 || mean_type > 6) return set_error(OMB_ERR_INVALID, "weighted mean type must be 1-6");
    if (mx < 0 || my < 0 || mz < 0 || mx > nx || my > ny || mz > nz)
        return set_error(OMB_ERR_INVALID, "weighted mean window must fit one mirror of the image");
    // types 4-6 read the image mirrored twice the window's reach
    if (mean_type >= 4 && (2 * mx > nx || 2 * my > ny || 2 * mz > nz))
        return set_error(OMB_ERR_INVALID, "weighted mean types 4-6 need twice the window within one mirror");
    if (!(wsum != 0.f)) return set_error(OMB_ERR_INVALID, "weighted mean weights sum to 0");
    // the reference takes a 2-D path for one slice (no z window)
    if (nz == 1 && mz > 0) return set_error(OMB_ERR_INVALID, "weighted mean of a single slice needs mz = 0");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    if (mean_type <= 3) {
        k_wmean_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, mx, my, mz, weights, wsum,
                                                                    mean_type, epps, beta, no_norm);
        OMB_LAUNCH_CHECK("weighted mean gradient launch");
        return OMB_OK;
    }
    const cudaStream_t st = (cudaStream_t)stream;
    const int ex = nx + 2 * mx, ey = ny + 2 * my, ez = nz + 2 * mz;
    if (ez > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    float *mext = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void **>(&mext), (size_t)ex * ey * ez * sizeof(float), st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(OMB_ERR_CUDA, "allocating the weighted means of types 4-6 failed");
    }
    dim3 gext((ex + 31) / 32, (ey + 7) / 8, ez);
    k_wmean_ext<<<gext, block, 0, st>>>(u, mext, nx, ny, nz, mx, my, mz, weights, wsum, mean_type);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        k_wmean_grad46<<<grid, block, 0, st>>>(u, mext, grad, nx, ny, nz, mx, my, mz, weights, mean_type, beta);
        e = cudaGetLastError();
    }
    cudaFreeAsync(mext, st);
    if (e != cudaSuccess) return set_error(OMB_ERR_CUDA, "weighted mean (types 4-6) launch failed");
    return OMB_OK;
}

namespace omb {

// Neighbour column c of the offsets grid the L-filter and FMH index
// (computeOffsets.m: ndgrid over -m..m on every axis, m = Ndx, x fastest;
// d = 3 axes, or 2 when Ndx + Ndy + Ndz < 3) as an offset (i, j, k).
__device__ __forceinline__ int3 nb_offset(int c, int m, int w, int d) {
    return make_int3(c % w - m, (c / w) % w - m, d == 3 ? c / (w * w) - m : 0);
}

__device__ __forceinline__ float mirrored(const float *__restrict__ u, int x, int y, int z, int3 o, int nx, int ny,
                                          int nz) {
    return __ldg(u + mirror(x + o.x, nx) + (int64_t)mirror(y + o.y, ny) * nx +
                 (int64_t)mirror(z + o.z, nz) * ((int64_t)nx * ny));
}

// L-filter prior (L_filter, priors.h:84-97): the w^d neighbourhood of the
// image mirrored at its faces sorted ascending, its weighted sum with a_L
// (a_L[r] weighs the value of rank r), grad += beta * (u - s) / (s + epps),
// or beta * (u - s) with no_norm.  Each value takes the weight of its rank
// (equal values share a rank range, and any split of it gives the same sum);
// one thread per voxel, the window in local memory (at most 125 values).
constexpr int kLfMax = 125;

__global__ void k_lfilter_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz, int m,
                                   int d, const float *__restrict__ a, float epps, float beta, int no_norm) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int w = 2 * m + 1;
    const int ncol = d == 3 ? w * w * w : w * w;
    float win[kLfMax];
    for (int c = 0; c < ncol; ++c) win[c] = mirrored(u, x, y, z, nb_offset(c, m, w, d), nx, ny, nz);
    float s = 0.f;
    for (int h = 0; h < ncol; ++h) {
        int rank = 0;
        for (int l = 0; l < ncol; ++l) rank += (win[l] < win[h] || (win[l] == win[h] && l < h)) ? 1 : 0;
        s = fmaf(__ldg(a + rank), win[h], s);
    }
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nx * ny;
    const float dv = __ldg(u + n) - s;
    grad[n] += no_norm ? dv * beta : dv / (s + epps) * beta;
}

// FMH prior (FMH, priors.h:54-82): nl lines through the voxel (13 in 3-D, 4
// when Nz = 1 or Ndz = 0), line ii the offsets-grid columns
// m ii + e (alku / m - ii), e = 0..2m, alku the centre column; each line's
// weighted mean with the column ii of fmh_weights ((2m+1) x nl, column-major
// as the reference loads it), the voxel's own value as value nl + 1, their
// median (the mean of the middle two for an even count, af::median);
// grad += beta * (u - med) / (med + epps), or beta * (u - med) with no_norm.
constexpr int kFmhLines = 13;

__global__ void k_fmh_gradient(const float *__restrict__ u, float *__restrict__ grad, int nx, int ny, int nz, int m,
                               int d, int nl, const float *__restrict__ fw, float epps, float beta, int no_norm) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const int w = 2 * m + 1;
    const int ncol = d == 3 ? w * w * w : w * w;
    const int step0 = (ncol - 1) / 2 / m;
    float v[kFmhLines + 1];
    for (int ii = 0; ii < nl; ++ii) {
        float acc = 0.f;
        for (int e = 0; e < w; ++e)
            acc = fmaf(__ldg(fw + e + ii * w), mirrored(u, x, y, z, nb_offset(m * ii + e * (step0 - ii), m, w, d), nx, ny, nz),
                       acc);
        v[ii] = acc;
    }
    const int64_t n = x + (int64_t)y * nx + (int64_t)z * nx * ny;
    const float un = __ldg(u + n);
    v[nl] = un;
    const int nv = nl + 1;
    for (int i = 1; i < nv; ++i) {
        const float t = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > t) {
            v[j + 1] = v[j];
            --j;
        }
        v[j + 1] = t;
    }
    const float med = (nv & 1) ? v[nv / 2] : 0.5f * (v[nv / 2 - 1] + v[nv / 2]);
    const float dv = un - med;
    grad[n] += no_norm ? dv * beta : dv / (med + epps) * beta;
}

// the offsets grids the reference's computeOffsets.m lays out consistently:
// Ndx = Ndy = Ndz (a cube, d = 3) or Ndx = Ndy = 1 with Ndz = 0 (d = 2)
static int median_filter_grid(int32_t nx, int32_t ny, int32_t nz, int32_t mx, int32_t my, int32_t mz, int max_m,
                              const char *what, int *d) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    const bool cube = mx >= 1 && mx <= max_m && my == mx && mz == mx;
    const bool square = mx == 1 && my == 1 && mz == 0;
    if (!cube && !square) return set_error(OMB_ERR_UNSUPPORTED, what);
    if (mx > nx || my > ny || mz > nz) return set_error(OMB_ERR_INVALID, "prior window larger than the image");
    *d = cube ? 3 : 2;
    return OMB_OK;
}

}  // namespace omb

extern "C" int omb_lfilter_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx,
                                    int32_t my, int32_t mz, const float *a_l, float epps, float beta, int32_t no_norm,
                                    void *stream) {
    using namespace omb;
    if (!u || !grad || !a_l) return set_error(OMB_ERR_INVALID, "u/grad/a_L pointer is NULL");
    int d = 0;
    const int st = median_filter_grid(nx, ny, nz, mx, my, mz, 2, "L-filter windows: Ndx = Ndy = Ndz <= 2, or Ndx = Ndy = 1 with Ndz = 0", &d);
    if (st != OMB_OK) return st;
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_lfilter_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, mx, d, a_l, epps, beta, no_norm);
    OMB_LAUNCH_CHECK("L-filter gradient launch");
    return OMB_OK;
}

extern "C" int omb_fmh_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx,
                                int32_t my, int32_t mz, const float *fmh_weights, float epps, float beta,
                                int32_t no_norm, void *stream) {
    using namespace omb;
    if (!u || !grad || !fmh_weights) return set_error(OMB_ERR_INVALID, "u/grad/fmh_weights pointer is NULL");
    int d = 0;
    const int st = median_filter_grid(nx, ny, nz, mx, my, mz, 8, "FMH windows: Ndx = Ndy = Ndz <= 8, or Ndx = Ndy = 1 with Ndz = 0", &d);
    if (st != OMB_OK) return st;
    const int nl = (nz == 1 || mz == 0) ? 4 : kFmhLines;
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    k_fmh_gradient<<<grid, block, 0, (cudaStream_t)stream>>>(u, grad, nx, ny, nz, mx, d, nl, fmh_weights, epps, beta,
                                                             no_norm);
    OMB_LAUNCH_CHECK("FMH gradient launch");
    return OMB_OK;
}
