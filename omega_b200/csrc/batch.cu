// Many independent small reconstructions in one persistent launch: a batch
// of CT geometries (e.g. 2-D fan-beam slices of different image sizes and
// view counts) projected by one improved-Siddon kernel.  The batch's rays are
// cut into chunks of 32 (one warp's rays); chunks of the largest items come
// first, and each warp takes the next chunk from a device counter until the
// list is exhausted, so uneven items keep every SM busy without one launch
// per item and no warp waits for the longest ray of its block.  Per-ray arithmetic is the type-1 projector's (siddon.cuh).
#include "kernels.h"
#include "siddon.cuh"

namespace omb {

// Chunks of 32 rays, one warp each: lane 0 takes the next chunk from the
// device counter and broadcasts it, so warps never wait for one another.
constexpr int kChunk = 32;

__device__ __forceinline__ int next_chunk(int *counter) {
    int v = 0;
    if ((threadIdx.x & 31) == 0) v = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, v, 0);
}

__global__ void __launch_bounds__(kBlock, 4) k_batch_fp(const BatchItem *__restrict__ items,
                                                        const int2 *__restrict__ work, int n_work,
                                                        int *__restrict__ counter, const float *__restrict__ img,
                                                        float *__restrict__ y) {
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    const int lane = threadIdx.x & 31;
    for (int wi = next_chunk(counter); wi < n_work; wi = next_chunk(counter)) {
        const int2 wk = work[wi];
        const BatchItem &it = items[wk.x];
        const int64_t r = (int64_t)wk.y + lane;
        if (r >= it.rs.m_size) continue;
        const float *im = img + it.img_off;
        const Ray ray = load_ray(it.rs, r);
        float temp = 0.f, ax = 0.f;
        const bool ok = siddon_walk<1, 4>(it.g, ray, false, 1.f, tof, temp,
                                          [&](int64_t ind, float ele, const float *, float) { ax += ele * __ldg(im + ind); });
        y[it.meas_off + r] = ok ? ax * temp : 0.f;
    }
}

__global__ void __launch_bounds__(kBlock) k_batch_bp(const BatchItem *__restrict__ items,
                                                     const int2 *__restrict__ work, int n_work,
                                                     int *__restrict__ counter, const float *__restrict__ y,
                                                     float *__restrict__ img) {
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    const int lane = threadIdx.x & 31;
    for (int wi = next_chunk(counter); wi < n_work; wi = next_chunk(counter)) {
        const int2 wk = work[wi];
        const BatchItem &it = items[wk.x];
        const int64_t r = (int64_t)wk.y + lane;
        if (r >= it.rs.m_size) continue;
        const float v = __ldg(y + it.meas_off + r);
        if (v == 0.f) continue;
        float *im = img + it.img_off;
        const Ray ray = load_ray(it.rs, r);
        float temp = 0.f;
        siddon_walk<1>(it.g, ray, false, 1.f, tof, temp, [&](int64_t ind, float ele, const float *, float) {
            const float c = ele * temp * v;
            if (c != 0.f) atomicAdd(im + ind, c);
        });
    }
}

int batch_project(const BatchItem *items, const int2 *work, int n_work, int *counter, const float *in, float *out,
                  bool backward, cudaStream_t st) {
    if (n_work <= 0) return OMB_OK;
    static int per_sm_fp = 0, per_sm_bp = 0;
    if (per_sm_fp == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_fp, k_batch_fp, kBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_bp, k_batch_bp, kBlock, 0);
        if (per_sm_fp < 1) per_sm_fp = 1;
        if (per_sm_bp < 1) per_sm_bp = 1;
    }
    OMB_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), st));
    const int per_sm = backward ? per_sm_bp : per_sm_fp;
    const int grid = min((n_work + kBlock / kChunk - 1) / (kBlock / kChunk), num_sms() * per_sm);
    if (backward)
        k_batch_bp<<<grid, kBlock, 0, st>>>(items, work, n_work, counter, in, out);
    else
        k_batch_fp<<<grid, kBlock, 0, st>>>(items, work, n_work, counter, in, out);
    OMB_LAUNCH_CHECK("batch projector launch");
    return OMB_OK;
}

}  // namespace omb
