// Projector type 1 (improved Siddon) forward and backprojection kernels.
//
// One thread per ray, grid-stride over the launch's rays in measurement order
// (detector row fastest), so a warp walks 32 neighbouring radial bins of one
// sinogram: coalesced float4 end-point loads and output stores, similar ray
// lengths inside the warp.  The image is gathered through the read-only
// cache (L2-resident for every image this path sees: 256 KiB-80 MiB).
#include "siddon.cuh"
#include "kernels.h"

namespace omb {

// Fixed-point scale of the deterministic backprojection: the reference's
// TH = 1e11 (omegatomo/projector/init.py:105).
constexpr double kFixedScale = 1e11;

template <int NB>
__global__ void __launch_bounds__(kBlock) k_siddon_fp(Grid g, RaySet rs, Tof tof, float gf,
                                                      const float *__restrict__ img, float *__restrict__ y) {
    const bool pet = rs.modality == OMB_PET_SINOGRAM;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        const Ray ray = load_ray(rs, r);
        float ax[NB];
#pragma unroll
        for (int to = 0; to < NB; ++to) ax[to] = 0.f;
        float temp = 0.f;
        const bool ok = siddon_walk<NB>(g, ray, pet, gf, tof, temp,
                                        [&](int64_t ind, float ele, const float *w, float tsum) {
                                            const float v = ele * __ldg(img + ind);
                                            if (NB == 1) {
                                                ax[0] += v;
                                            } else {
                                                const float dX = v / tsum;
#pragma unroll
                                                for (int to = 0; to < NB; ++to) ax[to] += w[to] * dX;
                                            }
                                        });
#pragma unroll
        for (int to = 0; to < NB; ++to) y[r + to * rs.m_size] = ok ? ax[to] * temp : 0.f;
    }
}

// Backprojection with float atomics (rhs(), general_opencl_functions.h:1212-1275).
template <int NB, bool SENS>
__global__ void __launch_bounds__(kBlock) k_siddon_bp(Grid g, RaySet rs, Tof tof, float gf,
                                                      const float *__restrict__ y, float *__restrict__ img,
                                                      float *__restrict__ sens) {
    const bool pet = rs.modality == OMB_PET_SINOGRAM;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        float ax[NB];
        bool any = SENS;
#pragma unroll
        for (int to = 0; to < NB; ++to) {
            ax[to] = y ? __ldg(y + r + to * rs.m_size) : 0.f;  // y == NULL: sensitivity only
            any |= ax[to] != 0.f;
        }
        if (!any) continue;  // adds only zeros
        const Ray ray = load_ray(rs, r);
        float temp = 0.f;
        siddon_walk<NB>(g, ray, pet, gf, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
            const float le = ele * temp;
            float yax, val;
            if (NB == 1) {
                yax = ax[0] * le;
                val = le;
                if (isnan(le)) yax = 0.f;
            } else {
                const float dX = le / tsum;
                yax = 0.f;
                val = 0.f;
#pragma unroll
                for (int to = 0; to < NB; ++to) {
                    const float a = dX * w[to];
                    val += a;
                    yax += a * ax[to];
                }
            }
            if (yax != 0.f) atomicAdd(img + ind, yax);
            if (SENS && val != 0.f) atomicAdd(sens + ind, val);
        });
    }
}

// Backprojection into int64 fixed point: every contribution is rounded to an
// integer on its own (toward zero, as OpenCL convert_long) and the integer
// sums are order independent, so the result is identical run to run.
// Semantics of the reference's -DATOMIC path (general_opencl_functions.h:1264-1272).
template <int NB, bool SENS>
__global__ void __launch_bounds__(kBlock) k_siddon_bp_fixed(Grid g, RaySet rs, Tof tof, float gf,
                                                            const float *__restrict__ y,
                                                            unsigned long long *__restrict__ acc,
                                                            unsigned long long *__restrict__ acc_sens) {
    const bool pet = rs.modality == OMB_PET_SINOGRAM;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        float ax[NB];
        bool any = SENS;
#pragma unroll
        for (int to = 0; to < NB; ++to) {
            ax[to] = __ldg(y + r + to * rs.m_size);
            any |= ax[to] != 0.f;
        }
        if (!any) continue;
        const Ray ray = load_ray(rs, r);
        float temp = 0.f;
        siddon_walk<NB>(g, ray, pet, gf, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
            const float le = ele * temp;
            float yax, val;
            if (NB == 1) {
                yax = ax[0] * le;
                val = le;
                if (isnan(le)) yax = 0.f;
            } else {
                const float dX = le / tsum;
                yax = 0.f;
                val = 0.f;
#pragma unroll
                for (int to = 0; to < NB; ++to) {
                    const float a = dX * w[to];
                    val += a;
                    yax += a * ax[to];
                }
            }
            const long long q = (long long)((double)yax * kFixedScale);
            if (q != 0) atomicAdd(acc + ind, (unsigned long long)q);
            if (SENS) {
                const long long qs = (long long)((double)val * kFixedScale);
                if (qs != 0) atomicAdd(acc_sens + ind, (unsigned long long)qs);
            }
        });
    }
}

__global__ void k_fixed_to_float(const unsigned long long *__restrict__ acc, float *__restrict__ out, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (float)((double)(long long)acc[i] * (1.0 / kFixedScale));
}

template <int NB>
static void fp_nb(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *img, float *y,
                  cudaStream_t st) {
    k_siddon_fp<NB><<<grid_for(rs.m_size), kBlock, 0, st>>>(g, rs, tof, gf, img, y);
}

template <int NB>
static void bp_nb(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y, float *img,
                  float *sens, unsigned long long *acc, unsigned long long *acc_sens, int mode, cudaStream_t st) {
    const unsigned grid = grid_for(rs.m_size);
    if (mode == OMB_BP_FIXED64) {
        if (acc_sens)
            k_siddon_bp_fixed<NB, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, acc, acc_sens);
        else
            k_siddon_bp_fixed<NB, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, acc, nullptr);
    } else {
        if (sens)
            k_siddon_bp<NB, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, img, sens);
        else
            k_siddon_bp<NB, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, img, nullptr);
    }
}

#define OMB_NB_CASES(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

int siddon_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *img, float *y,
                   cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    switch (tof.nbins) {
#define X(n) case n: fp_nb<n>(g, rs, tof, gf, img, y, st); break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("siddon forward launch");
    return OMB_OK;
}

int siddon_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y, float *img,
                    float *sens, unsigned long long *acc, unsigned long long *acc_sens, int mode,
                    cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    switch (tof.nbins) {
#define X(n) case n: bp_nb<n>(g, rs, tof, gf, y, img, sens, acc, acc_sens, mode, st); break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("siddon backward launch");
    return OMB_OK;
}

int fixed_to_float(const unsigned long long *acc, float *out, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_fixed_to_float<<<grid_for(n, 4), kBlock, 0, st>>>(acc, out, n);
    OMB_LAUNCH_CHECK("fixed-point conversion launch");
    return OMB_OK;
}

}  // namespace omb
