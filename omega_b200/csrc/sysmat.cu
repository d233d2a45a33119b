// Resident transposed system matrix of the improved-Siddon projector (type 1,
// non-TOF): the backprojection as a voxel-major gather instead of ray-driven
// atomics.
//
// The ray-driven backprojection adds y_r * a_rv to every voxel v its ray r
// crosses, with float atomics into L2 (for batched frames, float4 atomics of
// 4 frames at a time); on the dynamic-PET workload those atomics bound the
// kernel.  Here the weights a_rv of one subset -- the same walk, the same
// arithmetic (siddon_walk's crossing length x the ray's 1/L and correction
// factor) -- are computed once and stored voxel-major (for each voxel the
// (ray, weight) pairs of the rays crossing it, in ray order), 8 bytes a
// crossing, resident in HBM.  A backprojection is then one thread per voxel
// summing w * y over its list: no atomics, every voxel written once, and the
// sums taken in one fixed order (bit-identical call to call).  Frames are
// gathered 8 (or 4) at a time from a ray-major copy of the measurements
// (32 bytes a ray), so a crossing costs one 8-byte matrix read and one
// 32-byte gather for 8 frames.  Projector types 2 / 3 (non-TOF) build the
// same structure from the tube tracer's weights.
//
// After the build the lists are re-laid in slices of 32 consecutive voxels
// (one warp's voxels): entry k of every voxel of a slice side by side, so a
// warp reads its 32 matrix entries of step k as one 256-byte run instead of
// 32 scattered 8-byte reads.  Each voxel still sums its own list in ray
// order, so the result is the same bit for bit.
#include "common.cuh"
#include "kernels.h"
#include "siddon.cuh"

#include <vector>

namespace omb {
namespace {

// walks ray r and calls vis(voxel, weight) for each crossing the
// ray-driven backprojection would add to (finite, nonzero weight)
template <class Visit>
__device__ __forceinline__ void ray_weights(const Grid &g, const RaySet &rs, float gf, int64_t r, Visit &&vis) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    const Ray ray = load_ray(rs, r);
    const float gfr = pet && (rs.w || rs.mu) ? gf * ray_correction(g, rs, ray, r) : gf;
    float temp = 0.f;
    siddon_walk<1>(g, ray, pet, gfr, tof, temp, [&](int64_t ind, float ele, const float *, float) {
        const float le = ele * temp;
        if (isnan(le) || le == 0.f) return;
        vis(ind, le);
    });
}

__global__ void __launch_bounds__(kBlock) k_sm_count(Grid g, RaySet rs, float gf, unsigned *__restrict__ cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride)
        ray_weights(g, rs, gf, r, [&](int64_t ind, float) { atomicAdd(cnt + ind, 1u); });
}

__global__ void __launch_bounds__(kBlock) k_sm_fill(Grid g, RaySet rs, float gf,
                                                    unsigned long long *__restrict__ cursor, uint2 *__restrict__ ent) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride)
        ray_weights(g, rs, gf, r, [&](int64_t ind, float le) {
            const unsigned long long pos = atomicAdd(cursor + ind, 1ull);
            ent[pos] = make_uint2((unsigned)r, __float_as_uint(le));
        });
}

// Each voxel's list in ray order (the fill's atomics leave it in arrival
// order): insertion sort, one thread per voxel, once per build.
__global__ void k_sm_sort(const int64_t *__restrict__ off, uint2 *__restrict__ ent, int64_t n_img) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_img; v += stride) {
        const int64_t a = off[v], b = off[v + 1];
        for (int64_t i = a + 1; i < b; ++i) {
            const uint2 e = ent[i];
            int64_t k = i - 1;
            while (k >= a && ent[k].x > e.x) {
                ent[k + 1] = ent[k];
                --k;
            }
            ent[k + 1] = e;
        }
    }
}

// FB frames of the group starting at frame f0: ray-major copy, FB floats per ray
template <int FB>
__global__ void k_meas_to_raymajor(const float *__restrict__ meas, int64_t meas_stride, int nf, int64_t m,
                                   float *__restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += stride) {
        float v[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) v[f] = f < nf ? __ldg(meas + f * meas_stride + r) : 0.f;
        float4 *o = reinterpret_cast<float4 *>(out + r * FB);
#pragma unroll
        for (int q = 0; q < FB / 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
}

// One thread per voxel: img[f][v] = sum over its list of w * y[f][ray], in
// list order.  Neighbouring threads hold neighbouring voxels, whose lists
// share most of their rays in nearly the same positions, so a warp's gathers
// mostly meet lines already in L1.  FB = 4, 8: y ray-major (FB floats per
// ray); FB = 1: y read directly.
template <int FB>
__global__ void __launch_bounds__(kBlock) k_sm_bp(const int64_t *__restrict__ off, const uint2 *__restrict__ ent,
                                                  const float *__restrict__ y, int64_t n_img, float *__restrict__ img,
                                                  int64_t img_stride, int nf) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_img; v += stride) {
        float acc[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) acc[f] = 0.f;
        const int64_t a = __ldg(off + v), b = __ldg(off + v + 1);
#pragma unroll 4
        for (int64_t k = a; k < b; ++k) {
            const uint2 e = __ldg(ent + k);
            const float w = __uint_as_float(e.y);
            if (FB == 1) {
                acc[0] = fmaf(__ldg(y + e.x), w, acc[0]);
            } else {
                const float4 *p = reinterpret_cast<const float4 *>(y) + (int64_t)e.x * (FB / 4);
#pragma unroll
                for (int q = 0; q < FB / 4; ++q) {
                    const float4 t = __ldg(p + q);
                    acc[4 * q] = fmaf(t.x, w, acc[4 * q]);
                    acc[4 * q + 1] = fmaf(t.y, w, acc[4 * q + 1]);
                    acc[4 * q + 2] = fmaf(t.z, w, acc[4 * q + 2]);
                    acc[4 * q + 3] = fmaf(t.w, w, acc[4 * q + 3]);
                }
            }
        }
#pragma unroll
        for (int f = 0; f < FB; ++f)
            if (f < nf) img[f * img_stride + v] = acc[f];
    }
}

// the voxel-major lists re-laid in slices of 32 voxels (entry k of voxel l at soff[s] + 32 k + l)
__global__ void k_sm_slice(const int64_t *__restrict__ off, const uint2 *__restrict__ ent,
                           const int64_t *__restrict__ soff, uint2 *__restrict__ sent, int64_t n_img) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_img; v += stride) {
        const int64_t a = off[v], n = off[v + 1] - a;
        uint2 *d = sent + soff[v >> 5] + (v & 31);
        for (int64_t k = 0; k < n; ++k) d[k * 32] = ent[a + k];
    }
}

// k_sm_bp on the sliced lists: the grid-stride loop keeps a warp on the 32 voxels of one slice
template <int FB>
__global__ void __launch_bounds__(kBlock) k_sm_bp_sl(const int64_t *__restrict__ off, const int64_t *__restrict__ soff,
                                                     const uint2 *__restrict__ sent, const float *__restrict__ y,
                                                     int64_t n_img, float *__restrict__ img, int64_t img_stride, int nf) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_img; v += stride) {
        float acc[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) acc[f] = 0.f;
        const int64_t n = __ldg(off + v + 1) - __ldg(off + v);
        const uint2 *e0 = sent + __ldg(soff + (v >> 5)) + (v & 31);
#pragma unroll 4
        for (int64_t k = 0; k < n; ++k) {
            const uint2 e = __ldg(e0 + k * 32);
            const float w = __uint_as_float(e.y);
            if (FB == 1) {
                acc[0] = fmaf(__ldg(y + e.x), w, acc[0]);
            } else {
                const float4 *p = reinterpret_cast<const float4 *>(y) + (int64_t)e.x * (FB / 4);
#pragma unroll
                for (int q = 0; q < FB / 4; ++q) {
                    const float4 t = __ldg(p + q);
                    acc[4 * q] = fmaf(t.x, w, acc[4 * q]);
                    acc[4 * q + 1] = fmaf(t.y, w, acc[4 * q + 1]);
                    acc[4 * q + 2] = fmaf(t.z, w, acc[4 * q + 2]);
                    acc[4 * q + 3] = fmaf(t.w, w, acc[4 * q + 3]);
                }
            }
        }
#pragma unroll
        for (int f = 0; f < FB; ++f)
            if (f < nf) img[f * img_stride + v] = acc[f];
    }
}

// Forward projection through the ray-major slices: one thread per ray, y[r] = sum of w x[voxel] in the
// tracer's order (the grid-stride loop keeps a warp on the 32 rays of one slice)
__global__ void __launch_bounds__(kBlock) k_sm_fp_sl(const unsigned *__restrict__ rcnt,
                                                     const int64_t *__restrict__ rsoff, const uint2 *__restrict__ rsent,
                                                     const float *__restrict__ x, int64_t m, float *__restrict__ y) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += stride) {
        const unsigned n = __ldg(rcnt + r);
        const uint2 *e0 = rsent + __ldg(rsoff + (r >> 5)) + (r & 31);
        // two partial sums (even and odd entries) keep more loads in flight; fixed order, so the result
        // is the same call to call
        float acc0 = 0.f, acc1 = 0.f;
        unsigned k = 0;
#pragma unroll 4
        for (; k + 1 < n; k += 2) {
            const uint2 ea = __ldg(e0 + (int64_t)k * 32), eb = __ldg(e0 + (int64_t)(k + 1) * 32);
            acc0 = fmaf(__uint_as_float(ea.y), __ldg(x + ea.x), acc0);
            acc1 = fmaf(__uint_as_float(eb.y), __ldg(x + eb.x), acc1);
        }
        if (k < n) {
            const uint2 e = __ldg(e0 + (int64_t)k * 32);
            acc0 = fmaf(__uint_as_float(e.y), __ldg(x + e.x), acc0);
        }
        y[r] = acc0 + acc1;
    }
}

}  // namespace

int sysmat_forward(const Grid &g, const SysMat &sm, const Frames &fr, int64_t m, cudaStream_t st) {
    (void)g;
    if (!sm.rsent || !sm.rcnt) return set_error(OMB_ERR_INVALID, "system matrix has no forward copy");
    for (int f = 0; f < fr.n; ++f) {
        k_sm_fp_sl<<<grid_for(m, 8), kBlock, 0, st>>>(sm.rcnt, sm.rsoff, sm.rsent, fr.img_in + f * fr.img_stride, m,
                                                      fr.meas_out + f * fr.meas_stride);
        OMB_LAUNCH_CHECK("system matrix forward projection launch");
    }
    return OMB_OK;
}

void sysmat_free(SysMat &sm) {
    if (sm.off) cudaFree(sm.off);
    if (sm.ent) cudaFree(sm.ent);
    if (sm.soff) cudaFree(sm.soff);
    if (sm.sent) cudaFree(sm.sent);
    if (sm.rsoff) cudaFree(sm.rsoff);
    if (sm.rsent) cudaFree(sm.rsent);
    if (sm.rcnt) cudaFree(sm.rcnt);
    sm.off = nullptr;
    sm.ent = nullptr;
    sm.soff = nullptr;
    sm.sent = nullptr;
    sm.rsoff = nullptr;
    sm.rsent = nullptr;
    sm.rcnt = nullptr;
    sm.nnz = 0;
}

int sysmat_build(const Grid &g, const RaySet &rs, float gf, SysMat &sm, cudaStream_t st, const Orth *orth) {
    sysmat_free(sm);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return set_error(OMB_ERR_INVALID,
                         "the type-1 system matrix is built on the first backprojection of a subset, which must "
                         "not be captured into a CUDA graph (run one call first)");
    const int64_t n_img = (int64_t)g.nx * g.ny * g.nz;
    unsigned *cnt = nullptr;
    OMB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&cnt), (size_t)n_img * sizeof(unsigned), st));
    cudaMemsetAsync(cnt, 0, (size_t)n_img * sizeof(unsigned), st);
    unsigned *rcnt = nullptr;
    if (orth) {
        if (cudaMalloc(reinterpret_cast<void **>(&rcnt), (size_t)(rs.m_size > 0 ? rs.m_size : 1) * sizeof(unsigned)) !=
            cudaSuccess) {
            cudaGetLastError();
            cudaFreeAsync(cnt, st);
            return set_error(OMB_ERR_CUDA, "not enough device memory for the system matrix (ray counts)");
        }
        sm.rcnt = rcnt;
        const int ec = orth_sm_count(g, rs, *orth, gf, cnt, rcnt, st);
        if (ec != OMB_OK) {
            cudaFreeAsync(cnt, st);
            sysmat_free(sm);
            return ec;
        }
    } else {
        k_sm_count<<<grid_for(rs.m_size), kBlock, 0, st>>>(g, rs, gf, cnt);
    }
    std::vector<unsigned> hc((size_t)n_img);
    cudaMemcpyAsync(hc.data(), cnt, (size_t)n_img * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(cnt, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        sysmat_free(sm);
        return set_error(OMB_ERR_CUDA, "system matrix count pass failed");
    }
    std::vector<int64_t> ho((size_t)n_img + 1);
    ho[0] = 0;
    for (int64_t v = 0; v < n_img; ++v) ho[v + 1] = ho[v] + hc[v];
    const int64_t nnz = ho[n_img];
    std::vector<int64_t> hrs;
    if (orth) {
        // the ray-major copy's slice offsets (32 rays a slice, each slice as long as its longest ray)
        std::vector<unsigned> hr((size_t)rs.m_size);
        if (cudaMemcpy(hr.data(), rcnt, (size_t)rs.m_size * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) {
            sysmat_free(sm);
            return set_error(OMB_ERR_CUDA, "system matrix ray counts could not be read");
        }
        const int64_t n_sl = (rs.m_size + 31) / 32;
        hrs.assign((size_t)n_sl + 1, 0);
        for (int64_t s_ = 0; s_ < n_sl; ++s_) {
            unsigned mx = 0;
            for (int64_t r = s_ * 32; r < rs.m_size && r < s_ * 32 + 32; ++r) mx = hr[r] > mx ? hr[r] : mx;
            hrs[s_ + 1] = hrs[s_] + 32 * (int64_t)mx;
        }
        if (cudaMalloc(reinterpret_cast<void **>(&sm.rsoff), (size_t)(n_sl + 1) * sizeof(int64_t)) != cudaSuccess ||
            cudaMalloc(reinterpret_cast<void **>(&sm.rsent), (size_t)(hrs[n_sl] > 0 ? hrs[n_sl] : 1) * sizeof(uint2)) !=
                cudaSuccess) {
            // no room for the forward copy: the forward projection keeps the tracer
            cudaGetLastError();
            if (sm.rsoff) cudaFree(sm.rsoff);
            sm.rsoff = nullptr;
            sm.rsent = nullptr;
        } else {
            cudaMemcpy(sm.rsoff, hrs.data(), (size_t)(n_sl + 1) * sizeof(int64_t), cudaMemcpyHostToDevice);
        }
    }
    if (cudaMalloc(reinterpret_cast<void **>(&sm.off), (size_t)(n_img + 1) * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&sm.ent), (size_t)(nnz > 0 ? nnz : 1) * sizeof(uint2)) != cudaSuccess) {
        cudaGetLastError();
        sysmat_free(sm);
        return set_error(OMB_ERR_CUDA, "not enough device memory for the system matrix (" +
                                           std::to_string((double)nnz * 8.0 / 1e9) + " GB)");
    }
    cudaMemcpyAsync(sm.off, ho.data(), (size_t)(n_img + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
    unsigned long long *cursor = nullptr;
    OMB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&cursor), (size_t)n_img * sizeof(int64_t), st));
    cudaMemcpyAsync(cursor, sm.off, (size_t)n_img * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
    if (orth) {
        if (orth_sm_fill(g, rs, *orth, gf, cursor, sm.ent, sm.rsoff, sm.rsent, st) != OMB_OK) {
            cudaFreeAsync(cursor, st);
            sysmat_free(sm);
            return -1;
        }
    } else {
        k_sm_fill<<<grid_for(rs.m_size), kBlock, 0, st>>>(g, rs, gf, cursor, sm.ent);
    }
    k_sm_sort<<<grid_for(n_img), kBlock, 0, st>>>(sm.off, sm.ent, n_img);
    cudaFreeAsync(cursor, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        sysmat_free(sm);
        return set_error(OMB_ERR_CUDA, std::string("system matrix build failed: ") + cudaGetErrorString(e));
    }
    // the sliced copy: each slice as long as its longest list; kept only when it fits beside the lists
    {
        const int64_t n_sl = (n_img + 31) / 32;
        std::vector<int64_t> hs((size_t)n_sl + 1);
        hs[0] = 0;
        for (int64_t s_ = 0; s_ < n_sl; ++s_) {
            unsigned mx = 0;
            for (int64_t v = s_ * 32; v < n_img && v < s_ * 32 + 32; ++v) mx = hc[v] > mx ? hc[v] : mx;
            hs[s_ + 1] = hs[s_] + 32 * (int64_t)mx;
        }
        const int64_t tot = hs[n_sl];
        if (cudaMalloc(reinterpret_cast<void **>(&sm.soff), (size_t)(n_sl + 1) * sizeof(int64_t)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void **>(&sm.sent), (size_t)(tot > 0 ? tot : 1) * sizeof(uint2)) ==
                cudaSuccess) {
            cudaMemcpyAsync(sm.soff, hs.data(), (size_t)(n_sl + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
            k_sm_slice<<<grid_for(n_img), kBlock, 0, st>>>(sm.off, sm.ent, sm.soff, sm.sent, n_img);
            const cudaError_t e2 = cudaStreamSynchronize(st);
            if (e2 != cudaSuccess) {
                sysmat_free(sm);
                return set_error(OMB_ERR_CUDA, std::string("system matrix slicing failed: ") + cudaGetErrorString(e2));
            }
            cudaFree(sm.ent);
            sm.ent = nullptr;
        } else {
            // not enough memory for the copy: keep the lists
            cudaGetLastError();
            if (sm.soff) cudaFree(sm.soff);
            sm.soff = nullptr;
            sm.sent = nullptr;
        }
    }
    sm.nnz = nnz;
    sm.proj0 = rs.proj0;
    sm.m_size = rs.m_size;
    sm.cur_subset = rs.cur_subset;
    return OMB_OK;
}

int sysmat_backward(const Grid &g, const SysMat &sm, const Frames &fr, int64_t m, float *ym, int64_t ym_floats,
                    cudaStream_t st) {
    const int64_t n_img = (int64_t)g.nx * g.ny * g.nz;
    const int fb = fr.n >= 8 ? 8 : (fr.n >= 4 ? 4 : 1);
    if (fb > 1 && (!ym || ym_floats < fb * m))
        return set_error(OMB_ERR_INVALID, "system matrix backprojection: ray-major scratch too small");
    for (int f0 = 0; f0 < fr.n; f0 += fb) {
        const int nf = fr.n - f0 < fb ? fr.n - f0 : fb;
        const float *meas = fr.meas + f0 * fr.meas_stride;
        float *img = fr.img + f0 * fr.img_stride;
        const bool sl = sm.sent != nullptr;
        if (fb == 8) {
            k_meas_to_raymajor<8><<<grid_for(m, 4), kBlock, 0, st>>>(meas, fr.meas_stride, nf, m, ym);
            if (sl)
                k_sm_bp_sl<8><<<grid_for(n_img, 8), kBlock, 0, st>>>(sm.off, sm.soff, sm.sent, ym, n_img, img,
                                                                     fr.img_stride, nf);
            else
                k_sm_bp<8><<<grid_for(n_img, 8), kBlock, 0, st>>>(sm.off, sm.ent, ym, n_img, img, fr.img_stride, nf);
        } else if (fb == 4) {
            k_meas_to_raymajor<4><<<grid_for(m, 4), kBlock, 0, st>>>(meas, fr.meas_stride, nf, m, ym);
            if (sl)
                k_sm_bp_sl<4><<<grid_for(n_img, 8), kBlock, 0, st>>>(sm.off, sm.soff, sm.sent, ym, n_img, img,
                                                                     fr.img_stride, nf);
            else
                k_sm_bp<4><<<grid_for(n_img, 8), kBlock, 0, st>>>(sm.off, sm.ent, ym, n_img, img, fr.img_stride, nf);
        } else {
            if (sl)
                k_sm_bp_sl<1><<<grid_for(n_img, 8), kBlock, 0, st>>>(sm.off, sm.soff, sm.sent, meas, n_img, img,
                                                                     fr.img_stride, 1);
            else
                k_sm_bp<1><<<grid_for(n_img, 8), kBlock, 0, st>>>(sm.off, sm.ent, meas, n_img, img, fr.img_stride, 1);
        }
        OMB_LAUNCH_CHECK("system matrix backprojection launch");
    }
    return OMB_OK;
}

}  // namespace omb
