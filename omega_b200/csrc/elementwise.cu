// Elementwise and reduction steps of the OSEM subset update.
//
// ratio:  computeForwardProject.h:20-21 (input += epps), 92-95 (y / input),
//         400-401 (NaN/Inf -> epps)
// EM:     algorithms.h:12-15 via subiterStep.h:118-121 (im / Summ * (rhs + epps))
// clamp:  functions.hpp:2980-2996 (Summ < epps -> epps)
// All are HBM-bound streams: float4 loads/stores where the pointers allow.
#include "kernels.h"

namespace omb {

__device__ __forceinline__ float ratio1(float y, float f, float epps) {
    float r = y / (f + epps);
    if (isnan(r) || isinf(r)) r = epps;
    return r;
}

__global__ void k_osem_ratio(const float *__restrict__ y, float *__restrict__ fp, int64_t n, float epps) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t n4 = n / 4;
    const float4 *y4 = reinterpret_cast<const float4 *>(y);
    float4 *f4 = reinterpret_cast<float4 *>(fp);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        const float4 a = __ldg(y4 + i);
        float4 b = f4[i];
        b.x = ratio1(a.x, b.x, epps);
        b.y = ratio1(a.y, b.y, epps);
        b.z = ratio1(a.z, b.z, epps);
        b.w = ratio1(a.w, b.w, epps);
        f4[i] = b;
    }
    for (int64_t i = n4 * 4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        fp[i] = ratio1(y[i], fp[i], epps);
}

__global__ void k_em_update(float *__restrict__ img, const float *__restrict__ sens, const float *__restrict__ rhs,
                            int64_t n, float epps) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        img[i] = img[i] / __ldg(sens + i) * (__ldg(rhs + i) + epps);
}

__global__ void k_clamp_min(float *__restrict__ x, int64_t n, float lo) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (x[i] < lo) x[i] = lo;
}

// Frame batches: blockIdx.y selects the frame.
// With randoms (computeForwardProject.h:46-71): input = fp + epps + r, the
// ray's randoms shared by its TOF bins (bin stride n_rays).
__global__ void k_osem_ratio_randoms(const float *__restrict__ y, int64_t y_stride, float *__restrict__ fp,
                                     int64_t fp_stride, int64_t n, const float *__restrict__ rnd, int64_t n_rays,
                                     float epps) {
    const float *yf = y + blockIdx.y * y_stride;
    float *ff = fp + blockIdx.y * fp_stride;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float r = __ldg(yf + i) / ((ff[i] + epps) + __ldg(rnd + i % n_rays));
        if (isnan(r) || isinf(r)) r = epps;
        ff[i] = r;
    }
}

// One-step-late EM update (algorithms.h:24-27 OSL, subiterStep.h:219-226):
// x = x / (sens + dU) * rhs, dU the prior gradient (beta included).
__global__ void k_osl_update(float *__restrict__ img, const float *__restrict__ sens, const float *__restrict__ du,
                             const float *__restrict__ rhs, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        img[i] = img[i] / (__ldg(sens + i) + __ldg(du + i)) * __ldg(rhs + i);
}

int osl_update(float *img, const float *sens, const float *du, const float *rhs, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_osl_update<<<grid_for(n, 4), kBlock, 0, st>>>(img, sens, du, rhs, n);
    OMB_LAUNCH_CHECK("OSL update launch");
    return OMB_OK;
}

// du = beta * clamp(du, -delta, delta) (Huber_prior, priors.h:44-52; delta
// infinite for the quadratic prior)
__global__ void k_scale_clamp(float *__restrict__ du, int64_t n, float beta, float delta) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        du[i] = beta * fminf(fmaxf(du[i], -delta), delta);
}

int scale_clamp(float *du, int64_t n, float beta, float delta, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_scale_clamp<<<grid_for(n, 4), kBlock, 0, st>>>(du, n, beta, delta);
    OMB_LAUNCH_CHECK("prior scale launch");
    return OMB_OK;
}

// The relaxed updates (ROSEM algorithms.h:102-106; RAMLA / BSREM through
// PoissonUpdate, auxKernels.cl:1997-2026; the MAP step algorithms.h:130-135),
// the relaxation read per launch so that a captured iteration replays with
// the schedule's next value.
__device__ __forceinline__ float relax_value(const float *lam, const int *iter, float v) {
    return lam ? lam[*iter] : v;
}

__global__ void k_ratio_shift(const float *__restrict__ y, float *__restrict__ fp, int64_t n,
                              const float *__restrict__ rnd, int64_t n_rays, float epps, float shift, float sign) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float d = fp[i] + epps;
        if (rnd) d += __ldg(rnd + i % n_rays);
        float r = sign * (__ldg(y + i) / d - shift);
        if (isnan(r) || isinf(r)) r = epps;
        fp[i] = r;
    }
}

// PoissonUpdate, PKMA and MBSREM forms (auxKernels.cl:2008-2022)
// Image preconditioning of the gradient (applyImagePreconditioning,
// functions.hpp:2057-2106, types 0 and 1): 1 = g / D, 2 = g * (x_p / D) with
// x_p the image (PKMA) or min-folded image (MBSREM: U - x where x >= U / 2,
// algorithms.h:35-41); D the mean sensitivity over the subsets, 0 -> 1.
__device__ __forceinline__ float precondition(float g, int mode, const float *__restrict__ dd, int64_t i, float xp) {
    if (mode == 1) return g / __ldg(dd + i);
    if (mode == 2) return g * (xp / __ldg(dd + i));
    return g;
}

__global__ void k_pkma_update(float *__restrict__ img, const float *__restrict__ rhs, const float *__restrict__ du,
                              int64_t n, const float *__restrict__ lam_s, const int *__restrict__ it, float lam_v,
                              const float *__restrict__ al_s, int n_sub, int sub, float al_v, float epps,
                              int positivity, const float *__restrict__ dd, int mode) {
    const float lam = relax_value(lam_s, it, lam_v);
    const float a = al_s ? al_s[*it * n_sub + sub] : al_v;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = img[i];
        float g = du ? __ldg(rhs + i) + __ldg(du + i) : __ldg(rhs + i);
        g = precondition(g, mode, dd, i, x);
        float v = x - lam * g;
        if (positivity) v = fmaxf(epps, v);
        img[i] = (1.f - a) * x + a * v;
    }
}

__global__ void k_mbsrem_update(float *__restrict__ img, const float *__restrict__ rhs, const float *__restrict__ du,
                                int64_t n, const float *__restrict__ lam_s, const int *__restrict__ it, float lam_v,
                                float epps, float upper, int positivity, const float *__restrict__ dd, int mode) {
    const float lam = relax_value(lam_s, it, lam_v);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = img[i];
        float g = du ? __ldg(rhs + i) + __ldg(du + i) : __ldg(rhs + i);
        g = precondition(g, mode, dd, i, x >= upper / 2.f ? upper - x : x);
        float v = x + lam * g;
        if (positivity) v = fmaxf(epps, v);
        if (v >= upper) v = upper - epps;
        img[i] = v;
    }
}

// D = (sum of the subsets' sensitivities) / S, zeros -> 1 (reconstructionAF.h:779-816)
__global__ void k_precond_finish(float *__restrict__ dd, int64_t n, float subsets) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float v = dd[i];
        if (subsets > 1.f) v /= subsets;
        dd[i] = v == 0.f ? 1.f : v;
    }
}

__global__ void k_add_into(float *__restrict__ acc, const float *__restrict__ v, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) acc[i] += __ldg(v + i);
}

int precond_finish(float *dd, int64_t n, int subsets, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_precond_finish<<<grid_for(n, 4), kBlock, 0, st>>>(dd, n, (float)subsets);
    OMB_LAUNCH_CHECK("preconditioner image launch");
    return OMB_OK;
}

int add_into(float *acc, const float *v, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_add_into<<<grid_for(n, 4), kBlock, 0, st>>>(acc, v, n);
    OMB_LAUNCH_CHECK("image add launch");
    return OMB_OK;
}

__global__ void k_rosem_update(float *__restrict__ img, const float *__restrict__ sens, const float *__restrict__ rhs,
                               int64_t n, const float *__restrict__ lam_s, const int *__restrict__ it, float lam_v) {
    const float lam = relax_value(lam_s, it, lam_v);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = img[i], sm = __ldg(sens + i);
        img[i] = x + lam * x / sm * (__ldg(rhs + i) - sm);
    }
}

__global__ void k_bsrem_update(float *__restrict__ img, const float *__restrict__ rhs, int64_t n,
                               const float *__restrict__ lam_s, const int *__restrict__ it, float lam_v, float epps,
                               int positivity) {
    const float lam = relax_value(lam_s, it, lam_v);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = img[i];
        float v = x + lam * __ldg(rhs + i) * x;
        if (positivity) v = fmaxf(epps, v);
        img[i] = v;
    }
}

__global__ void k_map_step(float *__restrict__ img, const float *__restrict__ du, int64_t n,
                           const float *__restrict__ lam_s, const int *__restrict__ it, float lam_v, float epps) {
    const float lam = relax_value(lam_s, it, lam_v);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = img[i];
        const float v = x - lam * x * __ldg(du + i);
        img[i] = v < epps ? epps : v;
    }
}

__global__ void k_relax_advance(int *it) { *it += 1; }

int ratio_shift(const float *y, float *fp, int64_t n, const float *rnd, int64_t n_rays, float epps, float shift,
                float sign, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    if (rnd && n_rays <= 0) return set_error(OMB_ERR_INVALID, "randoms need n_rays > 0");
    k_ratio_shift<<<grid_for(n, 4), kBlock, 0, st>>>(y, fp, n, rnd, n_rays, epps, shift, sign);
    OMB_LAUNCH_CHECK("ratio launch");
    return OMB_OK;
}

int rosem_update(float *img, const float *sens, const float *rhs, int64_t n, Relax lam, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_rosem_update<<<grid_for(n, 4), kBlock, 0, st>>>(img, sens, rhs, n, lam.lam, lam.iter, lam.v);
    OMB_LAUNCH_CHECK("ROSEM update launch");
    return OMB_OK;
}

int bsrem_update(float *img, const float *rhs, int64_t n, Relax lam, float epps, bool positivity, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_bsrem_update<<<grid_for(n, 4), kBlock, 0, st>>>(img, rhs, n, lam.lam, lam.iter, lam.v, epps, positivity ? 1 : 0);
    OMB_LAUNCH_CHECK("BSREM update launch");
    return OMB_OK;
}

int pkma_update(float *img, const float *rhs, const float *du, int64_t n, Relax lam, Momentum a, float epps,
                bool positivity, const float *dd, int mode, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_pkma_update<<<grid_for(n, 4), kBlock, 0, st>>>(img, rhs, du, n, lam.lam, lam.iter, lam.v, a.alpha, a.n_subsets,
                                                     a.subset, a.v, epps, positivity ? 1 : 0, dd, mode);
    OMB_LAUNCH_CHECK("PKMA update launch");
    return OMB_OK;
}

int mbsrem_update(float *img, const float *rhs, const float *du, int64_t n, Relax lam, float epps, float upper,
                  bool positivity, const float *dd, int mode, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_mbsrem_update<<<grid_for(n, 4), kBlock, 0, st>>>(img, rhs, du, n, lam.lam, lam.iter, lam.v, epps, upper,
                                                       positivity ? 1 : 0, dd, mode);
    OMB_LAUNCH_CHECK("MBSREM update launch");
    return OMB_OK;
}

int map_step(float *img, const float *du, int64_t n, Relax lam, float epps, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_map_step<<<grid_for(n, 4), kBlock, 0, st>>>(img, du, n, lam.lam, lam.iter, lam.v, epps);
    OMB_LAUNCH_CHECK("MAP step launch");
    return OMB_OK;
}

int relax_advance(int *iter, cudaStream_t st) {
    k_relax_advance<<<1, 1, 0, st>>>(iter);
    OMB_LAUNCH_CHECK("relaxation counter launch");
    return OMB_OK;
}

int osem_ratio_randoms(const float *y, int64_t y_stride, float *fp, int64_t fp_stride, int64_t n, int frames,
                       const float *rnd, int64_t n_rays, float epps, cudaStream_t st) {
    if (n <= 0 || frames <= 0) return OMB_OK;
    if (frames > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 frames");
    dim3 grid((grid_for(n, 4) + frames - 1) / frames + 1, frames);
    k_osem_ratio_randoms<<<grid, kBlock, 0, st>>>(y, y_stride, fp, fp_stride, n, rnd, n_rays, epps);
    OMB_LAUNCH_CHECK("osem ratio launch");
    return OMB_OK;
}

__global__ void k_osem_ratio_frames(const float *__restrict__ y, int64_t y_stride, float *__restrict__ fp,
                                    int64_t fp_stride, int64_t n, float epps) {
    const float *yf = y + blockIdx.y * y_stride;
    float *ff = fp + blockIdx.y * fp_stride;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        ff[i] = ratio1(__ldg(yf + i), ff[i], epps);
}

__global__ void k_em_update_frames(float *__restrict__ img, int64_t img_stride, const float *__restrict__ sens,
                                   const float *__restrict__ rhs, int64_t rhs_stride, int64_t n, float epps) {
    float *xf = img + blockIdx.y * img_stride;
    const float *rf = rhs + blockIdx.y * rhs_stride;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        xf[i] = xf[i] / __ldg(sens + i) * (__ldg(rf + i) + epps);
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

int osem_ratio_frames(const float *y, int64_t y_stride, float *fp, int64_t fp_stride, int64_t n, int frames,
                      float epps, cudaStream_t st) {
    if (n <= 0 || frames <= 0) return OMB_OK;
    if (frames > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 frames");
    dim3 grid((grid_for(n, 4) + frames - 1) / frames + 1, frames);
    k_osem_ratio_frames<<<grid, kBlock, 0, st>>>(y, y_stride, fp, fp_stride, n, epps);
    OMB_LAUNCH_CHECK("osem ratio launch");
    return OMB_OK;
}

int em_update_frames(float *img, int64_t img_stride, const float *sens, const float *rhs, int64_t rhs_stride,
                     int64_t n, int frames, float epps, cudaStream_t st) {
    if (n <= 0 || frames <= 0) return OMB_OK;
    if (frames > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 frames");
    dim3 grid((grid_for(n, 4) + frames - 1) / frames + 1, frames);
    k_em_update_frames<<<grid, kBlock, 0, st>>>(img, img_stride, sens, rhs, rhs_stride, n, epps);
    OMB_LAUNCH_CHECK("EM update launch");
    return OMB_OK;
}

int osem_ratio(const float *y, float *fp, int64_t n, float epps, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    if (!aligned16(y) || !aligned16(fp)) return set_error(OMB_ERR_INVALID, "osem ratio buffers must be 16-byte aligned");
    k_osem_ratio<<<grid_for(n / 4 + 1, 4), kBlock, 0, st>>>(y, fp, n, epps);
    OMB_LAUNCH_CHECK("osem ratio launch");
    return OMB_OK;
}

int em_update(float *img, const float *sens, const float *rhs, int64_t n, float epps, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_em_update<<<grid_for(n, 4), kBlock, 0, st>>>(img, sens, rhs, n, epps);
    OMB_LAUNCH_CHECK("EM update launch");
    return OMB_OK;
}

int clamp_min(float *x, int64_t n, float lo, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_clamp_min<<<grid_for(n, 4), kBlock, 0, st>>>(x, n, lo);
    OMB_LAUNCH_CHECK("clamp launch");
    return OMB_OK;
}

// ---------------------------------------------------------------------------
// Poisson log-likelihood in FP64: two-pass block reduction (partials in the
// caller's workspace, then one block folds them), no atomics, so the result
// is identical run to run.
// ---------------------------------------------------------------------------

constexpr int kRedBlocks = 1184;  // 8 x 148 SMs

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = threadIdx.x < kBlock / 32 ? sh[threadIdx.x] : 0.0;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

__global__ void __launch_bounds__(kBlock) k_loglik_partial(const float *__restrict__ y, const float *__restrict__ fp,
                                                           int64_t n, float epps, double *__restrict__ part) {
    double acc = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double f = (double)__ldg(fp + i) + (double)epps;
        const double yy = (double)__ldg(y + i);
        acc += (yy != 0.0 ? yy * log(f) : 0.0) - f;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kBlock) k_sum_partials(const double *__restrict__ part, int n,
                                                         double *__restrict__ out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

size_t reduce_workspace_bytes(int64_t) { return (size_t)(kRedBlocks + 1) * sizeof(double); }

int loglik(const float *y, const float *fp, int64_t n, float epps, double *out_host, void *work, cudaStream_t st) {
    if (!work) return set_error(OMB_ERR_INVALID, "loglik workspace is NULL");
    if (!out_host) return set_error(OMB_ERR_INVALID, "loglik output pointer is NULL");
    double *part = static_cast<double *>(work);
    int blocks = (int)grid_for(n, 8);
    if (blocks > kRedBlocks) blocks = kRedBlocks;
    k_loglik_partial<<<blocks, kBlock, 0, st>>>(y, fp, n, epps, part);
    OMB_LAUNCH_CHECK("loglik partial launch");
    k_sum_partials<<<1, kBlock, 0, st>>>(part, blocks, part + kRedBlocks);
    OMB_LAUNCH_CHECK("loglik fold launch");
    OMB_CUDA_TRY(cudaMemcpyAsync(out_host, part + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, st));
    OMB_CUDA_TRY(cudaStreamSynchronize(st));
    return OMB_OK;
}

}  // namespace omb

// ---------------------------------------------------------------------------
// The other image preconditioners of PKMA / MRAMLA / MBSREM and PKMA's
// automatic relaxation (applyImagePreconditioning functions.hpp:2057-2106,
// gradientPreconditioner :2036-2054, computeGradient :2016-2035; PKMA
// algorithms.h:151-212).  The gradient g = rhs + dU is multiplied, in the
// reference's order, by the type-4 image gradF (from sub-iteration grad_init
// on), the type-3 value alpha[k], the types 0 / 1 / 2 factor (1 / D, xp / D,
// max(xp, max(1e-5, ref)) / D) and the type-6 image dP; xp is the image, for
// MBSREM folded to U - x where x >= U / 2.
// ---------------------------------------------------------------------------
namespace omb {
namespace {

__global__ void k_precond_apply(float *__restrict__ g, const float *__restrict__ du, const float *__restrict__ img,
                                int64_t n, PrecondExt p) {
    const int kk = *p.it * p.n_sub + p.sub;
    const bool grad = p.gradF && kk >= p.grad_init;
    const float al = p.alpha ? p.alpha[kk] : 1.f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = img[i];
        const float xp = p.fold && x >= p.upper / 2.f ? p.upper - x : x;
        float v = du ? g[i] + __ldg(du + i) : g[i];
        if (grad) v *= __ldg(p.gradF + i);
        if (p.alpha) v *= al;
        if (p.mode == 1) v /= __ldg(p.dd + i);
        else if (p.mode == 2) v *= xp / __ldg(p.dd + i);
        else if (p.mode == 3) v *= fmaxf(xp, fmaxf(1e-5f, __ldg(p.ref + i))) / __ldg(p.dd + i);
        if (p.dP) v *= __ldg(p.dP + i);
        g[i] = v;
    }
}

// deterministic FP64 sum in two passes (partials per block, then one block)
constexpr int kSumBlocks = 296;

// type-4 window check: sub-iteration k in [init, last]
__device__ __forceinline__ bool grad_window(const PrecondExt &p) {
    const int kk = *p.it * p.n_sub + p.sub;
    return kk >= p.grad_init && kk <= p.grad_last;
}

__device__ __forceinline__ float folded(const float *img, int64_t i, const PrecondExt &p) {
    const float x = img[i];
    return p.fold && x >= p.upper / 2.f ? p.upper - x : x;
}

// sum of the folded image (which = 0) or of gradF (which = 1) over the image
__global__ void k_grad_sum(const float *__restrict__ img, const float *__restrict__ f, int64_t n, PrecondExt p,
                           int which, double *__restrict__ part) {
    if (!grad_window(p)) return;
    __shared__ double sh[8];
    double acc = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        acc += which ? (double)__ldg(f + i) : (double)folded(img, i, p);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        part[blockIdx.x] = t;
    }
}

__global__ void k_grad_fold(double *__restrict__ part, int nb, PrecondExt p, double *__restrict__ out) {
    if (!grad_window(p)) return;
    double t = 0.0;
    for (int b = (int)threadIdx.x; b < nb; b += 32) t += part[b];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *out = t;
}

// one axis of computeGradient: forward (0), backward (1) or central (2)
// difference of the folded image at voxel (i along an axis of length len,
// neighbours at +-step)
__device__ __forceinline__ float axis_diff(const float *img, int64_t n0, int i, int len, int64_t step, int type,
                                           const PrecondExt &p) {
    const float c = folded(img, n0, p);
    if (type == 0) return i < len - 1 ? folded(img, n0 + step, p) - c : -c;
    if (type == 1) return i > 0 ? folded(img, n0 - step, p) - c : -c;
    if (len < 2) return 0.f;
    if (i == 0) return folded(img, n0 + step, p) - c;
    if (i == len - 1) return c - folded(img, n0 - step, p);
    return (folded(img, n0 + step, p) - folded(img, n0 - step, p)) * 0.5f;
}

// f = max(1e-5, |grad xp| / mean(xp)) into gradF
__global__ void k_grad_norm(const float *__restrict__ img, float *__restrict__ f, Grid g, PrecondExt p,
                            const double *__restrict__ sum_x) {
    if (!grad_window(p)) return;
    const int64_t nxy = (int64_t)g.nx * g.ny, n = nxy * g.nz;
    const float mean = (float)(*sum_x / (double)n);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const int k = (int)(v / nxy), j = (int)((v - k * nxy) / g.nx), i = (int)(v - k * nxy - (int64_t)j * g.nx);
        const float a = axis_diff(img, v, i, g.nx, 1, p.deriv_type, p);
        const float b = axis_diff(img, v, j, g.ny, g.nx, p.deriv_type, p);
        const float c = axis_diff(img, v, k, g.nz, nxy, p.deriv_type, p);
        f[v] = fmaxf(1e-5f, sqrtf(a * a + b * b + c * c) / mean);
    }
}

// gradF = min(V2, max(V1, mean(f) / f))
__global__ void k_grad_finish(float *__restrict__ f, int64_t n, PrecondExt p, const double *__restrict__ sum_f) {
    if (!grad_window(p)) return;
    const float mean = (float)(*sum_f / (double)n);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        f[v] = fminf(p.grad_v2, fmaxf(p.grad_v1, mean / f[v]));
}

// PKMA's relaxation (algorithms.h:155-197) from ||x||^2 and ||g||^2:
// first sub-iteration lam[0] = ||x|| / ||g|| / 4; first sub-iteration of
// iteration it > 0: lam[it] = lam[it - 1] / (it / 35 + 1); with scaling,
// q = ||x|| / (lam ||g||) and lam *= q / 1.5 when 0 < q < 1.5.
__global__ void k_pkma_relax(float *__restrict__ lam, const int *__restrict__ it, int sub, const double *xg_gg,
                             const double *gx_xx, int compute, int scaling) {
    const int t = *it;
    const double gn = sqrt(xg_gg[1]), xn = sqrt(gx_xx[1]);
    if (compute) {
        if (t == 0 && sub == 0) lam[0] = (float)(xn / gn) * .25f;
        else if (t > 0 && sub == 0) lam[t] = lam[t - 1] * (1.f / ((float)t / 35.f + 1.f));
    }
    if (scaling) {
        const float q = (float)(xn / (gn * (double)lam[t]));
        if (q < 1.5f && q > 0.f) lam[t] *= q / 1.5f;
    }
}

__global__ void k_div_inplace(float *__restrict__ a, const float *__restrict__ b, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] /= __ldg(b + i);
}

// E / y where y > 0, else 0 (the type-6 measurement image, reconstructionAF.h:600-616)
__global__ void k_curv_meas(float *__restrict__ e, const float *__restrict__ y, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float yv = __ldg(y + i);
        e[i] = yv > 0.f ? e[i] / yv : 0.f;
    }
}

// dP (+)= S / rhs; finish: NaN / Inf -> 1 (reconstructionAF.h:637-650)
__global__ void k_curv_acc(float *__restrict__ dp, const float *__restrict__ rhs, int64_t n, float S, int first) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float v = S / __ldg(rhs + i);
        dp[i] = first ? v : dp[i] + v;
    }
}

__global__ void k_curv_finish(float *__restrict__ dp, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (isnan(dp[i]) || isinf(dp[i])) dp[i] = 1.f;
}

// zeros of M -> 1 (reconstructionAF.h:861)
__global__ void k_zero_to_one(float *__restrict__ a, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (a[i] == 0.f) a[i] = 1.f;
}

}  // namespace

size_t precond_workspace_bytes() { return (size_t)(kSumBlocks + 2) * sizeof(double); }

int precond_apply(float *g, const float *du, const float *img, int64_t n, const PrecondExt &p, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_precond_apply<<<grid_for(n, 4), kBlock, 0, st>>>(g, du, img, n, p);
    OMB_LAUNCH_CHECK("image preconditioner launch");
    return OMB_OK;
}

int precond_gradient(const float *img, float *gradF, const Grid &g, const PrecondExt &p, double *work,
                     cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny * g.nz;
    double *part = work, *sx = work + kSumBlocks, *sf = work + kSumBlocks + 1;
    k_grad_sum<<<kSumBlocks, kBlock, 0, st>>>(img, nullptr, n, p, 0, part);
    k_grad_fold<<<1, 32, 0, st>>>(part, kSumBlocks, p, sx);
    k_grad_norm<<<grid_for(n, 4), kBlock, 0, st>>>(img, gradF, g, p, sx);
    k_grad_sum<<<kSumBlocks, kBlock, 0, st>>>(img, gradF, n, p, 1, part);
    k_grad_fold<<<1, 32, 0, st>>>(part, kSumBlocks, p, sf);
    k_grad_finish<<<grid_for(n, 4), kBlock, 0, st>>>(gradF, n, p, sf);
    OMB_LAUNCH_CHECK("gradient preconditioner launch");
    return OMB_OK;
}

int pkma_relax(float *lam, const int *it, int sub, const double *xg_gg, const double *gx_xx, bool compute,
               bool scaling, cudaStream_t st) {
    k_pkma_relax<<<1, 1, 0, st>>>(lam, it, sub, xg_gg, gx_xx, compute ? 1 : 0, scaling ? 1 : 0);
    OMB_LAUNCH_CHECK("PKMA relaxation launch");
    return OMB_OK;
}

int div_inplace(float *a, const float *b, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_div_inplace<<<grid_for(n, 4), kBlock, 0, st>>>(a, b, n);
    OMB_LAUNCH_CHECK("division launch");
    return OMB_OK;
}

int curv_meas(float *e, const float *y, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_curv_meas<<<grid_for(n, 4), kBlock, 0, st>>>(e, y, n);
    OMB_LAUNCH_CHECK("curvature preconditioner launch");
    return OMB_OK;
}

int curv_acc(float *dp, const float *rhs, int64_t n, int subsets, bool first, cudaStream_t st) {
    k_curv_acc<<<grid_for(n, 4), kBlock, 0, st>>>(dp, rhs, n, (float)subsets, first ? 1 : 0);
    OMB_LAUNCH_CHECK("curvature preconditioner launch");
    return OMB_OK;
}

int curv_finish(float *dp, int64_t n, cudaStream_t st) {
    k_curv_finish<<<grid_for(n, 4), kBlock, 0, st>>>(dp, n);
    OMB_LAUNCH_CHECK("curvature preconditioner launch");
    return OMB_OK;
}

int zero_to_one(float *a, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_zero_to_one<<<grid_for(n, 4), kBlock, 0, st>>>(a, n);
    OMB_LAUNCH_CHECK("measurement preconditioner launch");
    return OMB_OK;
}

}  // namespace omb
