// Multi-ray PET projection (the reference's N_RAYS option,
// projectorType123.cl:389-460, 779-840; CPU projector_functions.h:1441-1466,
// 2045-2058): every LOR is sampled by nr_xy x nr_z parallel rays spread over
// the crystal faces, each weighted 1 / (L_ray x rays) and walked by the
// improved Siddon traversal; the forward projection sums the rays, the
// backprojection spreads the measurement along each.  One thread per LOR, the
// rays walked one after the other (they hit the same voxels' neighbours, so
// the gathers stay in L1).
#include "siddon.cuh"
#include "kernels.h"

namespace omb {

template <int NB>
__global__ void __launch_bounds__(kBlock) k_siddon_fp_mr(Grid g, RaySet rs, Tof tof, float gf,
                                                         const float *__restrict__ img, float *__restrict__ y) {
    const int nrays = rs.nr_xy * rs.nr_z;
    const float gfn = gf / (float)nrays;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        const Ray base = load_ray(rs, r);
        float out[NB];
#pragma unroll
        for (int to = 0; to < NB; ++to) out[to] = 0.f;
        for (int lz = 0; lz < rs.nr_z; ++lz) {
            for (int lxy = 0; lxy < rs.nr_xy; ++lxy) {
                const Ray ray = multiray_shift(base, rs, lxy, lz);
                const float gfr = rs.w || rs.mu ? gfn * ray_correction(g, rs, ray, r) : gfn;
                float ax[NB];
#pragma unroll
                for (int to = 0; to < NB; ++to) ax[to] = 0.f;
                float temp = 0.f;
                const bool ok = siddon_walk<NB>(g, ray, true, gfr, tof, temp,
                                                [&](int64_t ind, float ele, const float *w, float tsum) {
                                                    if (NB == 1) {
                                                        ax[0] += ele * __ldg(img + ind);
                                                    } else {
                                                        const float dX = ele * __ldg(img + ind) / tsum;
#pragma unroll
                                                        for (int to = 0; to < NB; ++to) ax[to] += w[to] * dX;
                                                    }
                                                });
                if (ok) {
#pragma unroll
                    for (int to = 0; to < NB; ++to) out[to] += ax[to] * temp;
                }
            }
        }
#pragma unroll
        for (int to = 0; to < NB; ++to) y[r + to * rs.m_size] = out[to];
    }
}

template <int NB, bool SENS>
__global__ void __launch_bounds__(kBlock) k_siddon_bp_mr(Grid g, RaySet rs, Tof tof, float gf,
                                                         const float *__restrict__ y, float *__restrict__ img,
                                                         float *__restrict__ sens) {
    const int nrays = rs.nr_xy * rs.nr_z;
    const float gfn = gf / (float)nrays;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        float ax[NB];
        bool any = SENS;
#pragma unroll
        for (int to = 0; to < NB; ++to) {
            ax[to] = y ? __ldg(y + r + to * rs.m_size) : 0.f;
            any |= ax[to] != 0.f;
        }
        if (!any) continue;
        const Ray base = load_ray(rs, r);
        for (int lz = 0; lz < rs.nr_z; ++lz) {
            for (int lxy = 0; lxy < rs.nr_xy; ++lxy) {
                const Ray ray = multiray_shift(base, rs, lxy, lz);
                const float gfr = rs.w || rs.mu ? gfn * ray_correction(g, rs, ray, r) : gfn;
                float temp = 0.f;
                siddon_walk<NB>(g, ray, true, gfr, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
                    const float le = ele * temp;
                    float yax, val;
                    if (NB == 1) {
                        yax = isnan(le) ? 0.f : ax[0] * le;
                        val = le;
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
                    if (img && yax != 0.f) atomicAdd(img + ind, yax);
                    if (SENS && val != 0.f) atomicAdd(sens + ind, val);
                });
            }
        }
    }
}

#define OMB_NB_CASES(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

int multiray_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *img, float *y,
                     int per_sm, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    const unsigned grid = grid_for(rs.m_size, per_sm);
    switch (tof.nbins) {
#define X(n) case n: k_siddon_fp_mr<n><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, img, y); break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("multi-ray forward launch");
    return OMB_OK;
}

int multiray_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y, float *img,
                      float *sens, int per_sm, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    const unsigned grid = grid_for(rs.m_size, per_sm);
    switch (tof.nbins) {
#define X(n)                                                                                     \
    case n:                                                                                      \
        if (sens)                                                                                \
            k_siddon_bp_mr<n, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, img, sens);      \
        else                                                                                     \
            k_siddon_bp_mr<n, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, img, nullptr); \
        break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("multi-ray backward launch");
    return OMB_OK;
}

}  // namespace omb
