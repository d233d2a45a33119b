// Detector-row filtering of the filtering-based measurement preconditioner
// (applyMeasPreconditioning functions.hpp:2109-2166, filtering /
// filteringInverse :1882-1952): every detector column (nr rows, rows
// fastest) zero-padded to Nf, multiplied in the Fourier domain by a real,
// even filter, transformed back and cut to nr rows.  That is the circular
// convolution of the zero-padded column with h = ifft(filter) (real, even),
// computed here directly: out[i] = sum_{j < nr} h[(i - j) mod Nf] x[j].
//
// A CTA takes 16 columns: their nr x 16 values and the 2 nr - 1 taps
// e[k] = h[(k - nr + 1) mod Nf] are staged in shared memory; a thread owns 8
// consecutive rows x 4 columns and walks j with a sliding window of 8 taps in
// registers (one tap and 4 column values loaded per 32 multiply-adds).
#include "common.cuh"
#include "kernels.h"

namespace omb {
namespace {

constexpr int kCols = 16;  // columns per CTA
constexpr int kR = 8;      // rows per thread
constexpr int kC = 4;      // columns per thread
constexpr int kXS = 20;    // row stride of the staged columns (16-byte aligned, fewer bank conflicts)

__global__ void k_circ_filter(const float *__restrict__ in, float *__restrict__ out, int nr, int64_t ncols,
                              const float *__restrict__ h, int nf) {
    extern __shared__ float smem[];
    float *x = smem;                     // [nr][kXS]
    float *e = smem + (size_t)nr * kXS;  // [2 nr - 1] (+ kR padding)
    const int64_t col0 = (int64_t)blockIdx.x * kCols;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nt = blockDim.x * blockDim.y;
    for (int k = tid; k < 2 * nr - 1 + kR; k += nt) {
        const int d = k - (nr - 1);  // i - j
        e[k] = k < 2 * nr - 1 ? __ldg(h + ((d % nf) + nf) % nf) : 0.f;
    }
    for (int k = tid; k < nr * kCols; k += nt) {
        const int c = k / nr, r = k - c * nr;
        const int64_t col = col0 + c;
        x[r * kXS + c] = col < ncols ? __ldg(in + col * nr + r) : 0.f;
    }
    __syncthreads();
    const int c0 = threadIdx.x * kC;
    const int i0 = threadIdx.y * kR;
    if (i0 >= nr) return;
    float acc[kR][kC];
#pragma unroll
    for (int r = 0; r < kR; ++r)
#pragma unroll
        for (int c = 0; c < kC; ++c) acc[r][c] = 0.f;
    // taps of rows i0 + r at j = 0: e[i0 + r + nr - 1]
    float w[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) w[r] = e[i0 + r + nr - 1];
    for (int j = 0; j < nr; ++j) {
        const float4 xv = *reinterpret_cast<const float4 *>(x + j * kXS + c0);
#pragma unroll
        for (int r = 0; r < kR; ++r) {
            acc[r][0] = fmaf(w[r], xv.x, acc[r][0]);
            acc[r][1] = fmaf(w[r], xv.y, acc[r][1]);
            acc[r][2] = fmaf(w[r], xv.z, acc[r][2]);
            acc[r][3] = fmaf(w[r], xv.w, acc[r][3]);
        }
        // the taps for j + 1: index i - j - 1 + nr - 1
#pragma unroll
        for (int r = kR - 1; r > 0; --r) w[r] = w[r - 1];
        w[0] = e[i0 + nr - 2 - j >= 0 ? i0 + nr - 2 - j : 0];
    }
#pragma unroll
    for (int c = 0; c < kC; ++c) {
        const int64_t col = col0 + c0 + c;
        if (col >= ncols) continue;
#pragma unroll
        for (int r = 0; r < kR; ++r)
            if (i0 + r < nr) out[col * nr + i0 + r] = acc[r][c];
    }
}

}  // namespace

int circ_filter(const float *in, float *out, int nr, int64_t ncols, const float *h, int nf, cudaStream_t st) {
    if (nr < 1 || nr > 2048 || nf < nr) return set_error(OMB_ERR_INVALID, "row filter: 1 <= rows <= 2048 and Nf >= rows");
    if (ncols <= 0) return OMB_OK;
    const size_t smem = ((size_t)nr * kXS + 2 * (size_t)nr - 1 + kR) * sizeof(float);
    if (cudaFuncSetAttribute(k_circ_filter, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
        return set_error(OMB_ERR_CUDA, "row filter: shared memory attribute failed");
    dim3 block(kCols / kC, (nr + kR - 1) / kR);
    dim3 grid((unsigned)((ncols + kCols - 1) / kCols));
    k_circ_filter<<<grid, block, smem, st>>>(in, out, nr, ncols, h, nf);
    OMB_LAUNCH_CHECK("row filter launch");
    return OMB_OK;
}

}  // namespace omb

extern "C" int omb_row_filter(const float *in, float *out, int32_t n_rows, int64_t n_cols, const float *h, int32_t nf,
                              void *stream) {
    if (!in || !out || !h) return omb::set_error(OMB_ERR_INVALID, "NULL pointer passed to omb_row_filter");
    if (in == out) return omb::set_error(OMB_ERR_INVALID, "omb_row_filter: in and out must differ");
    return omb::circ_filter(in, out, n_rows, n_cols, h, nf, (cudaStream_t)stream);
}

namespace omb {
namespace {

__global__ void k_meas_residual(float *__restrict__ fp, const float *__restrict__ y, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) fp[i] -= __ldg(y + i);
}

// out = (p + sigma r) / denom (denom 1: no division)
__global__ void k_dual_step(const float *__restrict__ p, const float *__restrict__ r, float *__restrict__ out, int64_t n,
                            float sigma, float denom) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const bool divide = denom != 1.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float v = p[i] + sigma * __ldg(r + i);
        out[i] = divide ? v / denom : v;
    }
}

}  // namespace

int meas_residual(float *fp, const float *y, int64_t n, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_meas_residual<<<grid_for(n, 4), kBlock, 0, st>>>(fp, y, n);
    OMB_LAUNCH_CHECK("residual launch");
    return OMB_OK;
}

int dual_step(const float *p, const float *r, float *out, int64_t n, float sigma, float denom, cudaStream_t st) {
    if (n <= 0) return OMB_OK;
    k_dual_step<<<grid_for(n, 4), kBlock, 0, st>>>(p, r, out, n, sigma, denom);
    OMB_LAUNCH_CHECK("dual step launch");
    return OMB_OK;
}

}  // namespace omb
