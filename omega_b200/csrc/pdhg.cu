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

// ---------------------------------------------------------------------------
// The other TV gradients the reference compiles into TVKernel
// (auxKernels.cl:1733-1990), selected by TVtype / TV_use_anatomical / APLS
// (ProjectorClass.h:900-918, functions.hpp:1096-1113):
//   OMB_TV_SATV   TVtype 4 (SATV): per axis and side, d = u - neighbour,
//                 a = d / (|d| + epps); grad += beta sum (a - a / (|d| / sigma + 1))
//   OMB_TV_W1     TVtype 6 (TVW1): the plain TV's forward and backward
//                 differences weighted by exp(-(d / sigma)^2) per component
//   OMB_TV_ANAT1  anatomical TVtype 1: the quadratic forms of the 9-channel
//                 tensor S (prepass assembleS) on the same differences
//   OMB_TV_ANAT2  anatomical TVtype 2: the forward term's norm adds
//                 C |forward differences of the reference image S|^2
//   OMB_TV_APLS   anatomical TVtype 5 and APLS (C = eta): asymmetric parallel
//                 level sets with the reference image's normalised gradient
// The image is read edge-clamped (the texture path); S is read as zero past
// the last voxel (its buffer path).  The formulas keep the reference's own
// choices, e.g. TVW1's backward-z term weighted by w3.y and APLS's norms
// built from the raw reference gradient.
// ---------------------------------------------------------------------------
namespace omb {
namespace tvv {

struct Nb {
    float c, px, py, pz, mx, my, mz, uix, uiy, ujx, ujy, ukx, uky;
};

__device__ __forceinline__ Nb gather(const float *__restrict__ u, int i, int j, int k, int nx, int ny, int nz) {
    Nb b;
    b.c = tv_at(u, i, j, k, nx, ny, nz);
    b.px = tv_at(u, i + 1, j, k, nx, ny, nz);
    b.py = tv_at(u, i, j + 1, k, nx, ny, nz);
    b.pz = tv_at(u, i, j, k + 1, nx, ny, nz);
    b.mx = tv_at(u, i - 1, j, k, nx, ny, nz);
    b.my = tv_at(u, i, j - 1, k, nx, ny, nz);
    b.mz = tv_at(u, i, j, k - 1, nx, ny, nz);
    b.uix = tv_at(u, i - 1, j + 1, k, nx, ny, nz);
    b.uiy = tv_at(u, i - 1, j, k + 1, nx, ny, nz);
    b.ujx = tv_at(u, i + 1, j - 1, k, nx, ny, nz);
    b.ujy = tv_at(u, i, j - 1, k + 1, nx, ny, nz);
    b.ukx = tv_at(u, i + 1, j, k - 1, nx, ny, nz);
    b.uky = tv_at(u, i, j + 1, k - 1, nx, ny, nz);
    return b;
}

__device__ __forceinline__ float wnorm(float a, float b, float c, float wa, float wb, float wc, float eps) {
    return sqrtf(wa * a * a + wb * b * b + wc * c * c + eps);
}

__device__ __forceinline__ float w_of(float d, float sigma) {
    const float t = d / sigma;
    return __expf(-t * t);
}

}  // namespace tvv

template <int V>
__global__ void __launch_bounds__(256) k_tv_variant(const float *__restrict__ u, const float *__restrict__ S,
                                                    float *__restrict__ grad, int nx, int ny, int nz, float beta,
                                                    float eps, float sigma, float C) {
    using namespace tvv;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t nxy = (int64_t)nx * ny;
    const int64_t n = i + (int64_t)j * nx + (int64_t)k * nxy;
    const Nb b = gather(u, i, j, k, nx, ny, nz);
    // the backward-difference triples of the plain TV (u1, u2, u3)
    const float a1x = b.c - b.mx, a1y = b.uix - b.mx, a1z = b.uiy - b.mx;
    const float a2x = b.ujx - b.my, a2y = b.c - b.my, a2z = b.ujy - b.my;
    const float a3x = b.ukx - b.mz, a3y = b.uky - b.mz, a3z = b.c - b.mz;
    float g;
    if (V == OMB_TV_SATV) {
        const float d[6] = {b.c - b.px, b.c - b.mx, b.c - b.py, b.c - b.my, b.c - b.pz, b.c - b.mz};
        g = 0.f;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float ad = fabsf(d[q]);
            const float a = d[q] / (ad + eps);
            g += a - a / (ad / sigma + 1.f);
        }
    } else if (V == OMB_TV_W1) {
        const float fx = b.px - b.c, fy = b.py - b.c, fz = b.pz - b.c;
        const float w4x = w_of(fx, sigma), w4y = w_of(fy, sigma), w4z = w_of(fz, sigma);
        const float w1x = w_of(a1x, sigma), w1y = w_of(a1y, sigma), w1z = w_of(a1z, sigma);
        const float w2x = w_of(a2x, sigma), w2y = w_of(a2y, sigma), w2z = w_of(a2z, sigma);
        const float w3x = w_of(a3x, sigma), w3y = w_of(a3y, sigma), w3z = w_of(a3z, sigma);
        g = -(w4x * fx + w4y * fy + w4z * fz) / wnorm(fx, fy, fz, w4x, w4y, w4z, eps) +
            w1x * (b.c - b.mx) / wnorm(a1x, a1y, a1z, w1x, w1y, w1z, eps) +
            w2y * (b.c - b.my) / wnorm(a2x, a2y, a2z, w2x, w2y, w2z, eps) +
            w3y * (b.c - b.mz) / wnorm(a3x, a3y, a3z, w3x, w3y, w3z, eps);
    } else if (V == OMB_TV_ANAT1) {
        const int64_t N = nxy * nz;
        float s[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) s[q] = __ldg(S + n + q * N);
        auto pv = [&](float x, float y, float z) {
            return sqrtf(x * x * s[0] + y * y * s[4] + z * z * s[8] + (s[1] + s[3]) * x * y + (s[2] + s[6]) * x * z +
                         (s[5] + s[7]) * y * z + eps);
        };
        const float vx = b.px - b.c, vy = b.py - b.c, vz = b.pz - b.c;
        const float dx = s[0] * 2.f * (b.c - b.mx) + (s[3] + s[1]) * a1y + (s[2] + s[6]) * a1z;
        const float dy = s[4] * 2.f * (b.c - b.my) + (s[5] + s[7]) * a2z + (s[3] + s[1]) * a2x;
        const float dz = s[8] * 2.f * (b.c - b.mz) + (s[6] + s[2]) * a3x + (s[5] + s[7]) * a3y;
        const float d = (s[1] + s[2] + s[3] + s[6]) * vx + (s[1] + s[3] + s[5] + s[7]) * vy +
                        (s[2] + s[5] + s[6] + s[7]) * vz + 2.f * (s[0] * vx + s[4] * vy + s[8] * vz);
        g = 0.5f * (d / pv(vx, vy, vz) + dx / pv(a1x, a1y, a1z) + dy / pv(a2x, a2y, a2z) + dz / pv(a3x, a3y, a3z));
    } else {
        // anatomical types 2 and 5: forward differences of the reference image
        const float r0 = __ldg(S + n);
        const float rx = i < nx - 1 ? __ldg(S + n + 1) : 0.f;
        const float ry = j < ny - 1 ? __ldg(S + n + nx) : 0.f;
        const float rz = k < nz - 1 ? __ldg(S + n + nxy) : 0.f;
        const float fx = b.px - b.c, fy = b.py - b.c, fz = b.pz - b.c;
        if (V == OMB_TV_ANAT2) {
            const float sx = rx - r0, sy = ry - r0, sz = rz - r0;
            const float p0 = sqrtf(fx * fx + fy * fy + fz * fz + C * (sx * sx + sy * sy + sz * sz) + eps);
            g = (3.f * b.c - b.px - b.py - b.pz) / p0 + (b.c - b.mx) / wnorm(a1x, a1y, a1z, 1.f, 1.f, 1.f, eps) +
                (b.c - b.my) / wnorm(a2x, a2y, a2z, 1.f, 1.f, 1.f, eps) +
                (b.c - b.mz) / wnorm(a3x, a3y, a3z, 1.f, 1.f, 1.f, eps) + 1e-7f;
        } else {
            float ex = rx - r0, ey = ry - r0, ez = rz - r0;
            const float en = sqrtf(ex * ex + ey * ey + ez * ez + C * C);
            ex /= en;
            ey /= en;
            ez /= en;
            const float apuR = rx * fx + ry * fy + rz * fz;
            const float p0 = sqrtf(fx * fx + fy * fy + fz * fz - apuR * apuR + eps);
            auto pr = [&](float x, float y, float z) {
                const float rr = rx * x + ry * y + rz * z;
                return sqrtf(x * x + y * y + z * z + rr * rr + eps);
            };
            const float e1 = ex * a1x + ey * a1y + ez * a1z;
            const float e2 = ex * a2x + ey * a2y + ez * a2z;
            const float e3 = ex * a3x + ey * a3y + ez * a3z;
            const float ec = ex * (b.c - b.px) + ey * (b.c - b.py) + ez * (b.c - b.pz);
            g = 0.5f * ((6.f * b.c - 2.f * (b.px + b.py + b.pz) + 2.f * ec * (ex + ey + ez)) / p0 +
                        2.f * (a1x - ex * e1) / pr(a1x, a1y, a1z) + 2.f * (a2y - ey * e2) / pr(a2x, a2y, a2z) +
                        2.f * (a3z - ez * e3) / pr(a3x, a3y, a3z) + 1e-7f);
        }
    }
    grad[n] += beta * g;
}

}  // namespace omb

extern "C" int omb_tv_gradient_ex(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float beta,
                                  float smooth, int32_t variant, float sigma, float C, const float *ref,
                                  void *stream) {
    using namespace omb;
    if (variant == OMB_TV_PLAIN) return omb_tv_gradient(u, grad, nx, ny, nz, beta, smooth, stream);
    if (!u || !grad) return set_error(OMB_ERR_INVALID, "u/grad pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (variant < OMB_TV_SATV || variant > OMB_TV_APLS) return set_error(OMB_ERR_INVALID, "unknown TV variant");
    if (variant >= OMB_TV_ANAT1 && !ref)
        return set_error(OMB_ERR_INVALID, "anatomical TV and APLS need the reference image (or tensor)");
    if ((variant == OMB_TV_SATV || variant == OMB_TV_W1) && !(sigma != 0.f))
        return set_error(OMB_ERR_INVALID, "SATV and weighted TV need a nonzero sigma (SATVPhi)");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    cudaStream_t st = (cudaStream_t)stream;
#define OMB_TV_LAUNCH(V) k_tv_variant<V><<<grid, block, 0, st>>>(u, ref, grad, nx, ny, nz, beta, smooth, sigma, C)
    switch (variant) {
        case OMB_TV_SATV: OMB_TV_LAUNCH(OMB_TV_SATV); break;
        case OMB_TV_W1: OMB_TV_LAUNCH(OMB_TV_W1); break;
        case OMB_TV_ANAT1: OMB_TV_LAUNCH(OMB_TV_ANAT1); break;
        case OMB_TV_ANAT2: OMB_TV_LAUNCH(OMB_TV_ANAT2); break;
        default: OMB_TV_LAUNCH(OMB_TV_APLS); break;
    }
#undef OMB_TV_LAUNCH
    OMB_LAUNCH_CHECK("TV variant gradient launch");
    return OMB_OK;
}

// ---------------------------------------------------------------------------
// Proximal TV of the PDHG loop (priors.h:261-281; ProxTVGradient, ProxTVq,
// ProxTVDivergence auxKernels.cl:1141-1343).  The dual variable q holds three
// images (x, y, z components).  One step: q <- P_alpha(q + sigma2 D x), D the
// forward differences (DT 0; the last voxel's difference is -x) or the
// backward ones (DT 1; the first voxel's is x), P the projection onto the
// per-voxel L2 ball of radius alpha (L2) or the max-norm ball; then the
// primal right-hand side takes rhs -= div q, the sum of the backward (DT 0)
// or forward (DT 1) differences of the components.
// ---------------------------------------------------------------------------
namespace omb {

template <int DT, bool L2>
__global__ void __launch_bounds__(256) k_proxtv_dual(const float *__restrict__ x, float *__restrict__ q, int nx, int ny,
                                                     int nz, float sigma2, float alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t nxy = (int64_t)nx * ny, N = nxy * nz;
    const int64_t n = i + (int64_t)j * nx + (int64_t)k * nxy;
    const float c = __ldg(x + n);
    float gx, gy, gz;
    if (DT == 0) {
        gx = i < nx - 1 ? __ldg(x + n + 1) - c : -c;
        gy = j < ny - 1 ? __ldg(x + n + nx) - c : -c;
        gz = k < nz - 1 ? __ldg(x + n + nxy) - c : -c;
    } else {
        gx = i > 0 ? c - __ldg(x + n - 1) : c;
        gy = j > 0 ? c - __ldg(x + n - nx) : c;
        gz = k > 0 ? c - __ldg(x + n - nxy) : c;
    }
    // the scaled difference rounded before the addition, as the reference's kernel
    const float ax = q[n] + __fmul_rn(gx, sigma2);
    const float ay = q[n + N] + __fmul_rn(gy, sigma2);
    const float az = q[n + 2 * N] + __fmul_rn(gz, sigma2);
    const float scale = L2 ? fmaxf(1.f, sqrtf(ax * ax + ay * ay + az * az) / alpha)
                           : fmaxf(fmaxf(fabsf(az), fmaxf(fabsf(ax), fabsf(ay))) / alpha, 1.f);
    q[n] = ax / scale;
    q[n + N] = ay / scale;
    q[n + 2 * N] = az / scale;
}

template <int DT>
__global__ void __launch_bounds__(256) k_proxtv_div(const float *__restrict__ q, float *__restrict__ rhs, int nx, int ny,
                                                    int nz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t nxy = (int64_t)nx * ny, N = nxy * nz;
    const int64_t n = i + (int64_t)j * nx + (int64_t)k * nxy;
    const float *qx = q, *qy = q + N, *qz = q + 2 * N;
    float d = 0.f;
    if (DT == 0) {
        d += i > 0 ? __ldg(qx + n) - __ldg(qx + n - 1) : __ldg(qx + n);
        d += j > 0 ? __ldg(qy + n) - __ldg(qy + n - nx) : __ldg(qy + n);
        d += k > 0 ? __ldg(qz + n) - __ldg(qz + n - nxy) : __ldg(qz + n);
    } else {
        d += i < nx - 1 ? __ldg(qx + n + 1) - __ldg(qx + n) : -__ldg(qx + n);
        d += j < ny - 1 ? __ldg(qy + n + nx) - __ldg(qy + n) : -__ldg(qy + n);
        d += k < nz - 1 ? __ldg(qz + n + nxy) - __ldg(qz + n) : -__ldg(qz + n);
    }
    rhs[n] -= d;
}

}  // namespace omb

extern "C" int omb_proxtv_dual(const float *x, float *q, int32_t nx, int32_t ny, int32_t nz, float sigma2, float alpha,
                               int32_t l2_ball, int32_t diff_type, void *stream) {
    using namespace omb;
    if (!x || !q) return set_error(OMB_ERR_INVALID, "x/q pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (diff_type != 0 && diff_type != 1) return set_error(OMB_ERR_INVALID, "diff_type must be 0 or 1");
    if (!(alpha > 0.f)) return set_error(OMB_ERR_INVALID, "the proximal TV weight (beta) must be positive");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    cudaStream_t st = (cudaStream_t)stream;
    if (diff_type == 0) {
        if (l2_ball) k_proxtv_dual<0, true><<<grid, block, 0, st>>>(x, q, nx, ny, nz, sigma2, alpha);
        else k_proxtv_dual<0, false><<<grid, block, 0, st>>>(x, q, nx, ny, nz, sigma2, alpha);
    } else {
        if (l2_ball) k_proxtv_dual<1, true><<<grid, block, 0, st>>>(x, q, nx, ny, nz, sigma2, alpha);
        else k_proxtv_dual<1, false><<<grid, block, 0, st>>>(x, q, nx, ny, nz, sigma2, alpha);
    }
    OMB_LAUNCH_CHECK("proximal TV dual launch");
    return OMB_OK;
}

extern "C" int omb_proxtv_divergence(const float *q, float *rhs, int32_t nx, int32_t ny, int32_t nz, int32_t diff_type,
                                     void *stream) {
    using namespace omb;
    if (!q || !rhs) return set_error(OMB_ERR_INVALID, "q/rhs pointer is NULL");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (diff_type != 0 && diff_type != 1) return set_error(OMB_ERR_INVALID, "diff_type must be 0 or 1");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    cudaStream_t st = (cudaStream_t)stream;
    if (diff_type == 0) k_proxtv_div<0><<<grid, block, 0, st>>>(q, rhs, nx, ny, nz);
    else k_proxtv_div<1><<<grid, block, 0, st>>>(q, rhs, nx, ny, nz);
    OMB_LAUNCH_CHECK("proximal TV divergence launch");
    return OMB_OK;
}

// ---------------------------------------------------------------------------
// Proximal TGV of the PDHG loop (options.TGV; priors.h:284-313; ProxTVGradient
// with PROXTGV, ProxTVq, ProxTVDivergence, ProxTGVSymmDeriv, ProxTGVq,
// ProxTGVDivergence auxKernels.cl:1141-1560; forward differences):
//   q <- P_a0(q + sigma2 (D x - v)),  rhs -= div q,
//   r <- P_a1(r + sigma2 E v),  v1 = v + tau (q + div_sym r),  v <- v1 + theta (v1 - v).
// Z3: 3-D (v 3 images, r = (rxx, ryy, rzz, rxy, rxz, ryz)); else 2-D (v 2
// images, r = (rxx, ryy, rxy); the z difference of x enters q without v).
// ---------------------------------------------------------------------------
namespace omb {
namespace {

// forward difference of a (zero beyond the last voxel) at n along a stride
__device__ __forceinline__ float fwd_diff(const float *a, int64_t n, bool last, int64_t step) {
    const float c = __ldg(a + n);
    return last ? -c : __ldg(a + n + step) - c;
}

// backward difference (zero before the first voxel)
__device__ __forceinline__ float bwd_diff(const float *a, int64_t n, bool first, int64_t step) {
    const float c = __ldg(a + n);
    return first ? c : c - __ldg(a + n - step);
}

template <bool L2, bool Z3>
__global__ void __launch_bounds__(256) k_tgv_q(const float *__restrict__ x, const float *__restrict__ v,
                                               float *__restrict__ q, int nx, int ny, int nz, float sigma2,
                                               float alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t nxy = (int64_t)nx * ny, N = nxy * nz, n = i + (int64_t)j * nx + (int64_t)k * nxy;
    const float gx = fwd_diff(x, n, i == nx - 1, 1) - __ldg(v + n);
    const float gy = fwd_diff(x, n, j == ny - 1, nx) - __ldg(v + N + n);
    const float gz = Z3 ? fwd_diff(x, n, k == nz - 1, nxy) - __ldg(v + 2 * N + n) : fwd_diff(x, n, k == nz - 1, nxy);
    const float ax = q[n] + __fmul_rn(gx, sigma2), ay = q[n + N] + __fmul_rn(gy, sigma2);
    const float az = q[n + 2 * N] + __fmul_rn(gz, sigma2);
    const float scale = L2 ? fmaxf(1.f, sqrtf(ax * ax + ay * ay + az * az) / alpha)
                           : fmaxf(fmaxf(fabsf(az), fmaxf(fabsf(ax), fabsf(ay))) / alpha, 1.f);
    q[n] = ax / scale;
    q[n + N] = ay / scale;
    q[n + 2 * N] = az / scale;
}

template <bool L2, bool Z3>
__global__ void __launch_bounds__(256) k_tgv_r(const float *__restrict__ v, float *__restrict__ r, int nx, int ny,
                                               int nz, float sigma2, float alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t nxy = (int64_t)nx * ny, N = nxy * nz, n = i + (int64_t)j * nx + (int64_t)k * nxy;
    const bool lx = i == nx - 1, ly = j == ny - 1, lz = k == nz - 1;
    const float *vx = v, *vy = v + N, *vz = v + 2 * N;
    const float h = __fmul_rn(sigma2, .5f);
    if (Z3) {
        float d[6];
        d[0] = r[n] + __fmul_rn(fwd_diff(vx, n, lx, 1), sigma2);
        d[1] = r[n + N] + __fmul_rn(fwd_diff(vy, n, ly, nx), sigma2);
        d[2] = r[n + 2 * N] + __fmul_rn(fwd_diff(vz, n, lz, nxy), sigma2);
        d[3] = r[n + 3 * N] + __fmul_rn(fwd_diff(vx, n, ly, nx) + fwd_diff(vy, n, lx, 1), h);
        d[4] = r[n + 4 * N] + __fmul_rn(fwd_diff(vx, n, lz, nxy) + fwd_diff(vz, n, lx, 1), h);
        d[5] = r[n + 5 * N] + __fmul_rn(fwd_diff(vy, n, lz, nxy) + fwd_diff(vz, n, ly, nx), h);
        const float scale =
            L2 ? fmaxf(1.f, sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] +
                                  2.f * (d[3] * d[3]) + 2.f * (d[4] * d[4]) + 2.f * (d[5] * d[5])) / alpha)
               : fmaxf(fmaxf(fabsf(d[5]), fmaxf(fabsf(d[4]), fmaxf(fabsf(d[3]), fmaxf(fabsf(d[2]),
                                                                                       fmaxf(fabsf(d[0]), fabsf(d[1])))))) /
                           alpha,
                       1.f);
#pragma unroll
        for (int c = 0; c < 6; ++c) r[n + c * N] = d[c] / scale;
    } else {
        float d[3];
        d[0] = r[n] + __fmul_rn(fwd_diff(vx, n, lx, 1), sigma2);
        d[1] = r[n + N] + __fmul_rn(fwd_diff(vy, n, ly, nx), sigma2);
        d[2] = r[n + 2 * N] + __fmul_rn(fwd_diff(vx, n, ly, nx) + fwd_diff(vy, n, lx, 1), h);
        const float scale = L2 ? fmaxf(1.f, sqrtf(d[0] * d[0] + d[1] * d[1] + 2.f * (d[2] * d[2])) / alpha)
                               : fmaxf(fmaxf(fabsf(d[2]), fmaxf(fabsf(d[0]), fabsf(d[1]))) / alpha, 1.f);
#pragma unroll
        for (int c = 0; c < 3; ++c) r[n + c * N] = d[c] / scale;
    }
}

template <bool Z3>
__global__ void __launch_bounds__(256) k_tgv_v(const float *__restrict__ r, const float *__restrict__ q,
                                               float *__restrict__ v, int nx, int ny, int nz, float theta, float tau) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const int64_t nxy = (int64_t)nx * ny, N = nxy * nz, n = i + (int64_t)j * nx + (int64_t)k * nxy;
    const bool fx = i == 0, fy = j == 0, fz = k == 0;
    float dv[3];
    if (Z3) {
        dv[0] = bwd_diff(r, n, fx, 1) + bwd_diff(r + 3 * N, n, fy, nx) + bwd_diff(r + 4 * N, n, fz, nxy);
        dv[1] = bwd_diff(r + N, n, fy, nx) + bwd_diff(r + 3 * N, n, fx, 1) + bwd_diff(r + 5 * N, n, fz, nxy);
        dv[2] = bwd_diff(r + 2 * N, n, fz, nxy) + bwd_diff(r + 4 * N, n, fx, 1) + bwd_diff(r + 5 * N, n, fy, nx);
    } else {
        dv[0] = bwd_diff(r, n, fx, 1) + bwd_diff(r + 2 * N, n, fy, nx);
        dv[1] = bwd_diff(r + N, n, fy, nx) + bwd_diff(r + 2 * N, n, fx, 1);
    }
#pragma unroll
    for (int c = 0; c < (Z3 ? 3 : 2); ++c) {
        const float vo = v[n + c * N];
        const float v1 = fmaf(tau, __ldg(q + n + c * N) + dv[c], vo);
        v[n + c * N] = fmaf(theta, v1 - vo, v1);
    }
}

}  // namespace
}  // namespace omb

extern "C" int omb_proxtgv_step(const float *x, float *q, float *r, float *v, float *rhs, int32_t nx, int32_t ny,
                                int32_t nz, float sigma2, float alpha0, float alpha1, float theta, float tau,
                                int32_t l2_ball, int32_t three_d, void *stream) {
    using namespace omb;
    if (!x || !q || !r || !v || !rhs) return set_error(OMB_ERR_INVALID, "NULL pointer passed to omb_proxtgv_step");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    if (!(alpha0 > 0.f) || !(alpha1 > 0.f)) return set_error(OMB_ERR_INVALID, "the TGV weights alpha0, alpha1 must be positive");
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8, nz);
    cudaStream_t st = (cudaStream_t)stream;
#define OMB_TGV(L, Z)                                                                         \
    k_tgv_q<L, Z><<<grid, block, 0, st>>>(x, v, q, nx, ny, nz, sigma2, alpha0);               \
    k_proxtv_div<0><<<grid, block, 0, st>>>(q, rhs, nx, ny, nz);                              \
    k_tgv_r<L, Z><<<grid, block, 0, st>>>(v, r, nx, ny, nz, sigma2, alpha1);                  \
    k_tgv_v<Z><<<grid, block, 0, st>>>(r, q, v, nx, ny, nz, theta, tau);
    if (l2_ball && three_d) {
        OMB_TGV(true, true)
    } else if (l2_ball) {
        OMB_TGV(true, false)
    } else if (three_d) {
        OMB_TGV(false, true)
    } else {
        OMB_TGV(false, false)
    }
#undef OMB_TGV
    OMB_LAUNCH_CHECK("proximal TGV launch");
    return OMB_OK;
}
