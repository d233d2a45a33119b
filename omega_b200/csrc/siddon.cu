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

// Forward projection.  Each thread walks one ray once and accumulates it for
// FB frames of a dynamic study (blockIdx.y selects the group of frames), so
// the traversal cost is shared by up to FB images.  Non-TOF forward walks are
// latency-bound gathers: capping them at 64 registers (4 blocks, 32 warps per
// SM) beats the spills it costs (measured: 30.6 -> 23.6 ms single-frame, 6.0
// -> 3.9 ms for the interleaved 8-frame walk); the TOF variants keep their
// registers (their weight arrays would spill hundreds of bytes).
template <int NB, int FB, typename T, int K>
__global__ void __launch_bounds__(kBlock, NB == 1 ? 4 : 1) k_siddon_fp(Grid g, RaySet rs, Tof tof, float gf,
                                                      const T *__restrict__ img, int64_t img_stride,
                                                      float *__restrict__ y, int64_t y_stride, int n_frames) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const int f0 = blockIdx.y * FB;
    const int nf = min(FB, n_frames - f0);
    img += f0 * img_stride;
    y += f0 * y_stride;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        const Ray ray = load_ray(rs, r);
        const float gfr = pet && (rs.w || rs.mu) ? gf * ray_correction(g, rs, ray, r) : gf;
        float ax[NB * FB];
#pragma unroll
        for (int to = 0; to < NB * FB; ++to) ax[to] = 0.f;
        float temp = 0.f;
        const bool ok = siddon_walk<NB, K>(g, ray, pet, gfr, tof, temp,
                                        [&](int64_t ind, float ele, const float *w, float tsum) {
                                            if (NB == 1) {
#pragma unroll
                                                for (int f = 0; f < FB; ++f)
                                                    if (f < nf) ax[f] += ele * ld_img(img + f * img_stride + ind);
                                            } else {
                                                const float dX = ele * ld_img(img + ind) / tsum;
#pragma unroll
                                                for (int to = 0; to < NB; ++to) ax[to] += w[to] * dX;
                                            }
                                        });
        if (NB == 1) {
#pragma unroll
            for (int f = 0; f < FB; ++f)
                if (f < nf) y[f * y_stride + r] = ok ? ax[f] * temp : 0.f;
        } else {
#pragma unroll
            for (int to = 0; to < NB; ++to) y[r + to * rs.m_size] = ok ? ax[to] * temp : 0.f;
        }
    }
}

// Voxel-interleaved frame batches.  A group of FB (4 or 8) frames is stored
// as one run of FB floats per voxel, [group][voxel][frame], so the forward
// walk reads all FB values of an intersected voxel with FB/4 16-byte loads
// (one 32-byte sector for FB = 8) instead of FB scattered 4-byte gathers, and
// the backprojection updates them with FB/4 vector atomics (float4 atomicAdd,
// sm_90+) instead of FB scalar ones.  Frames past the batch's end are zero.
template <int FB>
__global__ void __launch_bounds__(kBlock) k_frames_interleave(const float *__restrict__ img, int64_t img_stride,
                                                              int n_frames, int64_t n, float *__restrict__ out) {
    const int f0 = blockIdx.y * FB;
    const int nf = min(FB, n_frames - f0);
    float4 *o = reinterpret_cast<float4 *>(out + (int64_t)blockIdx.y * n * FB);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        float a[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) a[f] = f < nf ? __ldg(img + (f0 + f) * img_stride + v) : 0.f;
#pragma unroll
        for (int q = 0; q < FB / 4; ++q) o[v * (FB / 4) + q] = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
    }
}

template <int FB>
__global__ void __launch_bounds__(kBlock) k_frames_deinterleave(const float *__restrict__ in, int n_frames, int64_t n,
                                                                float *__restrict__ img, int64_t img_stride) {
    const int f0 = blockIdx.y * FB;
    const int nf = min(FB, n_frames - f0);
    const float4 *p = reinterpret_cast<const float4 *>(in + (int64_t)blockIdx.y * n * FB);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        float a[FB];
#pragma unroll
        for (int q = 0; q < FB / 4; ++q) {
            const float4 t = __ldg(p + v * (FB / 4) + q);
            a[4 * q] = t.x;
            a[4 * q + 1] = t.y;
            a[4 * q + 2] = t.z;
            a[4 * q + 3] = t.w;
        }
#pragma unroll
        for (int f = 0; f < FB; ++f)
            if (f < nf) img[(f0 + f) * img_stride + v] = a[f];
    }
}

template <int FB, int K>
__global__ void __launch_bounds__(kBlock, 4) k_siddon_fp_ilv(Grid g, RaySet rs, float gf, const float *__restrict__ img,
                                                          int64_t n_img, float *__restrict__ y, int64_t y_stride,
                                                          int n_frames) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    const int f0 = blockIdx.y * FB;
    const int nf = min(FB, n_frames - f0);
    const float4 *im = reinterpret_cast<const float4 *>(img + (int64_t)blockIdx.y * n_img * FB);
    y += f0 * y_stride;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        const Ray ray = load_ray(rs, r);
        const float gfr = pet && (rs.w || rs.mu) ? gf * ray_correction(g, rs, ray, r) : gf;
        float ax[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) ax[f] = 0.f;
        float temp = 0.f;
        const bool ok = siddon_walk<1, K>(g, ray, pet, gfr, tof, temp, [&](int64_t ind, float ele, const float *, float) {
#pragma unroll
            for (int q = 0; q < FB / 4; ++q) {
                const float4 t = __ldg(im + ind * (FB / 4) + q);
                ax[4 * q] += ele * t.x;
                ax[4 * q + 1] += ele * t.y;
                ax[4 * q + 2] += ele * t.z;
                ax[4 * q + 3] += ele * t.w;
            }
        });
#pragma unroll
        for (int f = 0; f < FB; ++f)
            if (f < nf) y[f * y_stride + r] = ok ? ax[f] * temp : 0.f;
    }
}

template <int FB>
__global__ void __launch_bounds__(kBlock) k_siddon_bp_ilv(Grid g, RaySet rs, float gf, const float *__restrict__ y,
                                                          int64_t y_stride, float *__restrict__ img, int64_t n_img,
                                                          int n_frames) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    const int f0 = blockIdx.y * FB;
    const int nf = min(FB, n_frames - f0);
    y += f0 * y_stride;
    float4 *im = reinterpret_cast<float4 *>(img + (int64_t)blockIdx.y * n_img * FB);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // the next ray's measurements and end points are loaded before this
    // ray's walk, so their latency hides behind it
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float axn[FB];
    Ray rayn{};
    if (r < rs.m_size) {
#pragma unroll
        for (int f = 0; f < FB; ++f) axn[f] = f < nf ? __ldg(y + f * y_stride + r) : 0.f;
        rayn = load_ray(rs, r);
    }
    for (; r < rs.m_size; r += stride) {
        float ax[FB];
        bool any = false;
#pragma unroll
        for (int f = 0; f < FB; ++f) {
            ax[f] = axn[f];
            any |= ax[f] != 0.f;
        }
        const Ray ray = rayn;
        const int64_t rn = r + stride;
        if (rn < rs.m_size) {
#pragma unroll
            for (int f = 0; f < FB; ++f) axn[f] = f < nf ? __ldg(y + f * y_stride + rn) : 0.f;
            rayn = load_ray(rs, rn);
        }
        if (!any) continue;  // adds only zeros
        const float gfr = pet && (rs.w || rs.mu) ? gf * ray_correction(g, rs, ray, r) : gf;
        float temp = 0.f;
        siddon_walk<1>(g, ray, pet, gfr, tof, temp, [&](int64_t ind, float ele, const float *, float) {
            const float le = ele * temp;
            if (isnan(le) || le == 0.f) return;
#pragma unroll
            for (int q = 0; q < FB / 4; ++q) {
                const float4 c = make_float4(ax[4 * q] * le, ax[4 * q + 1] * le, ax[4 * q + 2] * le, ax[4 * q + 3] * le);
                if (c.x != 0.f || c.y != 0.f || c.z != 0.f || c.w != 0.f) atomicAdd(im + ind * (FB / 4) + q, c);
            }
        });
    }
}

// Backprojection with float atomics (rhs(), general_opencl_functions.h:1212-1275).
// Frame batching as in the forward kernel: one walk, FB images updated.
template <int NB, int FB, bool SENS>
__global__ void __launch_bounds__(kBlock) k_siddon_bp(Grid g, RaySet rs, Tof tof, float gf,
                                                      const float *__restrict__ y, int64_t y_stride,
                                                      float *__restrict__ img, int64_t img_stride,
                                                      float *__restrict__ sens, int n_frames) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const int f0 = blockIdx.y * FB;
    const int nf = min(FB, n_frames - f0);
    if (y) y += f0 * y_stride;
    if (img) img += f0 * img_stride;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        float ax[NB * FB];
        bool any = SENS;
        if (NB == 1) {
#pragma unroll
            for (int f = 0; f < FB; ++f) {
                ax[f] = (y && f < nf) ? __ldg(y + f * y_stride + r) : 0.f;  // y == NULL: sensitivity only
                any |= ax[f] != 0.f;
            }
        } else {
#pragma unroll
            for (int to = 0; to < NB; ++to) {
                ax[to] = y ? __ldg(y + r + to * rs.m_size) : 0.f;
                any |= ax[to] != 0.f;
            }
        }
        if (!any) continue;  // adds only zeros
        const Ray ray = load_ray(rs, r);
        const float gfr = pet && (rs.w || rs.mu) ? gf * ray_correction(g, rs, ray, r) : gf;
        float temp = 0.f;
        siddon_walk<NB>(g, ray, pet, gfr, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
            const float le = ele * temp;
            if (NB == 1) {
                if (!isnan(le)) {
#pragma unroll
                    for (int f = 0; f < FB; ++f) {
                        const float yax = ax[f] * le;
                        if (f < nf && yax != 0.f) atomicAdd(img + f * img_stride + ind, yax);
                    }
                }
                if (SENS && le != 0.f) atomicAdd(sens + ind, le);
            } else {
                const float dX = le / tsum;
                float yax = 0.f, val = 0.f;
#pragma unroll
                for (int to = 0; to < NB; ++to) {
                    const float a = dX * w[to];
                    val += a;
                    yax += a * ax[to];
                }
                if (yax != 0.f) atomicAdd(img + ind, yax);
                if (SENS && val != 0.f) atomicAdd(sens + ind, val);
            }
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
    const bool pet = rs.modality != OMB_CT_PANEL;
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
        const float gfr = pet && (rs.w || rs.mu) ? gf * ray_correction(g, rs, ray, r) : gf;
        float temp = 0.f;
        siddon_walk<NB>(g, ray, pet, gfr, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
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

// Voxel intersections Np summed over the launch's rays (the walk lengths of
// the algorithmic-byte model); one int64 atomic per block.
__global__ void __launch_bounds__(kBlock) k_siddon_count(Grid g, RaySet rs, Tof tof,
                                                         unsigned long long *__restrict__ total) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long n = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        const Ray ray = load_ray(rs, r);
        float temp;
        siddon_walk<1>(g, ray, pet, 1.f, tof, temp, [&](int64_t, float, const float *, float) { ++n; });
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    __shared__ unsigned long long sh[kBlock / 32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kBlock / 32; ++i) t += sh[i];
        atomicAdd(total, t);
    }
}

int siddon_count(const Grid &g, const RaySet &rs, const Tof &tof, unsigned long long *total, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    Tof t1 = tof;
    t1.nbins = 1;
    k_siddon_count<<<grid_for(rs.m_size), kBlock, 0, st>>>(g, rs, t1, total);
    OMB_LAUNCH_CHECK("siddon count launch");
    return OMB_OK;
}

__global__ void k_fixed_to_float(const unsigned long long *__restrict__ acc, float *__restrict__ out, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (float)((double)(long long)acc[i] * (1.0 / kFixedScale));
}

template <int NB, int FB, int K>
static void fp_launch_k(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, int per_sm,
                        cudaStream_t st) {
    dim3 grid(grid_for(rs.m_size, per_sm), (fr.n + FB - 1) / FB);
    if (fr.img_in16)
        k_siddon_fp<NB, FB, __nv_bfloat16, K><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, fr.img_in16, fr.img_stride,
                                                                       fr.meas_out, fr.meas_stride, fr.n);
    else
        k_siddon_fp<NB, FB, float, K><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, fr.img_in, fr.img_stride, fr.meas_out,
                                                               fr.meas_stride, fr.n);
}

// k: crossings taken per batched walk step (1, 2, 4; TOF walks take 1)
template <int NB, int FB>
static void fp_launch(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, int per_sm, int k,
                      cudaStream_t st) {
    if constexpr (NB == 1) {
        if (k == 4) return fp_launch_k<NB, FB, 4>(g, rs, tof, gf, fr, per_sm, st);
        if (k == 2) return fp_launch_k<NB, FB, 2>(g, rs, tof, gf, fr, per_sm, st);
    }
    fp_launch_k<NB, FB, 1>(g, rs, tof, gf, fr, per_sm, st);
}

template <int NB, int FB>
static void bp_launch(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, float *sens,
                      int per_sm, cudaStream_t st) {
    dim3 grid(grid_for(rs.m_size, per_sm), (fr.n + FB - 1) / FB);
    if (sens)
        k_siddon_bp<NB, FB, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, fr.meas, fr.meas_stride, fr.img,
                                                             fr.img_stride, sens, fr.n);
    else
        k_siddon_bp<NB, FB, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, fr.meas, fr.meas_stride, fr.img,
                                                              fr.img_stride, nullptr, fr.n);
}

template <int NB>
static void bp_fixed_launch(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y,
                            unsigned long long *acc, unsigned long long *acc_sens, cudaStream_t st) {
    const unsigned grid = grid_for(rs.m_size);
    if (acc_sens)
        k_siddon_bp_fixed<NB, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, acc, acc_sens);
    else
        k_siddon_bp_fixed<NB, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, y, acc, nullptr);
}

#define OMB_NB_CASES(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

// Frames per walk for non-TOF batches (at most `most`).
static int frames_per_walk(int n, int most) {
    n = n < most ? n : most;
    return n >= 8 ? 8 : (n >= 4 ? 4 : (n >= 2 ? 2 : 1));
}

// Frames per walk of the voxel-interleaved path (4 or 8), or 0 when the batch
// takes the frame-major kernels.
static int interleaved_frames(const Tof &tof, const Frames &fr, const Tuning &tn, int64_t n_img) {
    if (tn.siddon_layout != 1 || tof.nbins != 1 || !fr.ilv || fr.img_in16) return 0;
    const int fb = frames_per_walk(fr.n, tn.siddon_frames);
    if (fb < 4) return 0;
    const int64_t groups = (fr.n + fb - 1) / fb;
    return groups * fb * n_img <= fr.ilv_floats ? fb : 0;
}

template <int FB>
static void fp_ilv_launch(const Grid &g, const RaySet &rs, float gf, const Frames &fr, int64_t n_img, int per_sm,
                          int k, cudaStream_t st) {
    const unsigned groups = (fr.n + FB - 1) / FB;
    k_frames_interleave<FB><<<dim3(grid_for(n_img, 4), groups), kBlock, 0, st>>>(fr.img_in, fr.img_stride, fr.n,
                                                                                  n_img, fr.ilv);
    const dim3 grid(grid_for(rs.m_size, per_sm), groups);
    if (k == 4)
        k_siddon_fp_ilv<FB, 4><<<grid, kBlock, 0, st>>>(g, rs, gf, fr.ilv, n_img, fr.meas_out, fr.meas_stride, fr.n);
    else if (k == 2)
        k_siddon_fp_ilv<FB, 2><<<grid, kBlock, 0, st>>>(g, rs, gf, fr.ilv, n_img, fr.meas_out, fr.meas_stride, fr.n);
    else
        k_siddon_fp_ilv<FB, 1><<<grid, kBlock, 0, st>>>(g, rs, gf, fr.ilv, n_img, fr.meas_out, fr.meas_stride, fr.n);
}

template <int FB>
static int bp_ilv_launch(const Grid &g, const RaySet &rs, float gf, const Frames &fr, int64_t n_img, int per_sm,
                         cudaStream_t st) {
    const unsigned groups = (fr.n + FB - 1) / FB;
    OMB_CUDA_TRY(cudaMemsetAsync(fr.ilv, 0, (size_t)groups * FB * n_img * sizeof(float), st));
    k_siddon_bp_ilv<FB><<<dim3(grid_for(rs.m_size, per_sm), groups), kBlock, 0, st>>>(g, rs, gf, fr.meas,
                                                                                        fr.meas_stride, fr.ilv, n_img, fr.n);
    k_frames_deinterleave<FB><<<dim3(grid_for(n_img, 4), groups), kBlock, 0, st>>>(fr.ilv, fr.n, n_img, fr.img,
                                                                                    fr.img_stride);
    return OMB_OK;
}

int siddon_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, const Tuning &tn,
                   cudaStream_t st) {
    const int ps = tn.siddon_blocks_per_sm;
    if (rs.m_size <= 0 || fr.n <= 0) return OMB_OK;
    if (tof.nbins > 1 && fr.n != 1) return set_error(OMB_ERR_UNSUPPORTED, "TOF projections take one frame per call");
    const int64_t n_img = (int64_t)g.nx * g.ny * g.nz;
    const int ilv = interleaved_frames(tof, fr, tn, n_img);
    const int k = tn.siddon_fp_steps;
    if (ilv == 8) {
        fp_ilv_launch<8>(g, rs, gf, fr, n_img, ps, k, st);
    } else if (ilv == 4) {
        fp_ilv_launch<4>(g, rs, gf, fr, n_img, ps, k, st);
    } else if (tof.nbins == 1) {
        switch (frames_per_walk(fr.n, tn.siddon_frames)) {
            case 8: fp_launch<1, 8>(g, rs, tof, gf, fr, ps, k, st); break;
            case 4: fp_launch<1, 4>(g, rs, tof, gf, fr, ps, k, st); break;
            case 2: fp_launch<1, 2>(g, rs, tof, gf, fr, ps, k, st); break;
            default: fp_launch<1, 1>(g, rs, tof, gf, fr, ps, k, st); break;
        }
    } else {
        switch (tof.nbins) {
#define X(n) case n: fp_launch<n, 1>(g, rs, tof, gf, fr, ps, 1, st); break;
            OMB_NB_CASES(X)
#undef X
            default:
                return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
        }
    }
    OMB_LAUNCH_CHECK("siddon forward launch");
    return OMB_OK;
}

int siddon_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, float *sens,
                    const Tuning &tn, cudaStream_t st) {
    const int ps = tn.siddon_blocks_per_sm;
    if (rs.m_size <= 0 || fr.n <= 0) return OMB_OK;
    if (tof.nbins > 1 && fr.n != 1) return set_error(OMB_ERR_UNSUPPORTED, "TOF projections take one frame per call");
    const int64_t n_img = (int64_t)g.nx * g.ny * g.nz;
    // the interleaved kernels write every voxel of every frame (no sensitivity)
    const int ilv = sens || !fr.meas || !fr.img ? 0 : interleaved_frames(tof, fr, tn, n_img);
    if (ilv == 8) {
        const int e = bp_ilv_launch<8>(g, rs, gf, fr, n_img, ps, st);
        if (e != OMB_OK) return e;
    } else if (ilv == 4) {
        const int e = bp_ilv_launch<4>(g, rs, gf, fr, n_img, ps, st);
        if (e != OMB_OK) return e;
    } else if (tof.nbins == 1) {
        switch (frames_per_walk(fr.n, tn.siddon_frames)) {
            case 8: bp_launch<1, 8>(g, rs, tof, gf, fr, sens, ps, st); break;
            case 4: bp_launch<1, 4>(g, rs, tof, gf, fr, sens, ps, st); break;
            case 2: bp_launch<1, 2>(g, rs, tof, gf, fr, sens, ps, st); break;
            default: bp_launch<1, 1>(g, rs, tof, gf, fr, sens, ps, st); break;
        }
    } else {
        switch (tof.nbins) {
#define X(n) case n: bp_launch<n, 1>(g, rs, tof, gf, fr, sens, ps, st); break;
            OMB_NB_CASES(X)
#undef X
            default:
                return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
        }
    }
    OMB_LAUNCH_CHECK("siddon backward launch");
    return OMB_OK;
}

int siddon_backward_fixed(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y,
                          unsigned long long *acc, unsigned long long *acc_sens, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    switch (tof.nbins) {
#define X(n) case n: bp_fixed_launch<n>(g, rs, tof, gf, y, acc, acc_sens, st); break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("siddon fixed-point backward launch");
    return OMB_OK;
}

int fixed_to_float(const unsigned long long *acc, float *out, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_fixed_to_float<<<grid_for(n, 4), kBlock, 0, st>>>(acc, out, n);
    OMB_LAUNCH_CHECK("fixed-point conversion launch");
    return OMB_OK;
}

}  // namespace omb
