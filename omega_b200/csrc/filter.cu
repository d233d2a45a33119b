// Detector-row filtering of the filtering-based measurement preconditioner
// (applyMeasPreconditioning functions.hpp:2109-2166, filtering /
// filteringInverse :1882-1952): every detector column (nr rows, rows
// fastest) zero-padded to Nf, multiplied in the Fourier domain by a real,
// even filter, transformed back and cut to nr rows.  That is the circular
// convolution of the zero-padded column with h = ifft(filter) (real, even),
// computed here directly: out[i] = sum_{j < nr} h[(i - j) mod Nf] x[j].
//
// The same kernel filters the image lines of the filtering-based image
// preconditioner (filtering2D functions.hpp:1908-1932: every slice
// zero-padded to Nf x Nf, multiplied by the separable filter f f^T / max,
// cut back): x lines, then y lines, each a circular convolution with the
// 1-D taps scaled by 1 / sqrt(max).
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

// Where element (row r, column c) of the filtered data lies: (c % cdim) * cs0 + (c / cdim) * cs1 + r * rs.
// Detector columns: rs = 1, cs0 = rows, cdim = columns.  Image x lines: rs = 1, cs0 = nx, cdim = ny nz.
// Image y lines: rs = nx, cs0 = 1, cdim = nx, cs1 = nx ny.
struct Lines {
    int64_t rs, cs0, cs1, cdim;
    __device__ __forceinline__ int64_t at(int64_t c, int r) const { return (c % cdim) * cs0 + (c / cdim) * cs1 + r * rs; }
};

// the gate of a filter inside a replayed loop: active in sub-iteration kk = *it * n_sub + sub when kk < K
// (K > 0) or kk == 0 (K == 0); always active without a counter
__device__ __forceinline__ bool gate_open(const FilterGate &g) {
    if (!g.it) return true;
    const int kk = *g.it * g.n_sub + g.sub;
    return g.K > 0 ? kk < g.K : kk == 0;
}

__global__ void k_circ_filter(const float *__restrict__ in, float *__restrict__ out, int nr, int64_t ncols, Lines L,
                              const float *__restrict__ h, int nf, FilterGate gate) {
    if (!gate_open(gate)) return;
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
    if (L.rs == 1) {
        // rows contiguous: consecutive threads take consecutive rows
        for (int k = tid; k < nr * kCols; k += nt) {
            const int c = k / nr, r = k - c * nr;
            const int64_t col = col0 + c;
            x[r * kXS + c] = col < ncols ? __ldg(in + L.at(col, r)) : 0.f;
        }
    } else {
        // columns contiguous: consecutive threads take consecutive columns
        for (int k = tid; k < nr * kCols; k += nt) {
            const int r = k / kCols, c = k - r * kCols;
            const int64_t col = col0 + c;
            x[r * kXS + c] = col < ncols ? __ldg(in + L.at(col, r)) : 0.f;
        }
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
            if (i0 + r < nr) out[L.at(col, i0 + r)] = acc[r][c];
    }
}

}  // namespace

namespace {
int launch_lines(const float *in, float *out, int nr, int64_t ncols, const Lines &L, const float *h, int nf,
                 const FilterGate &gate, cudaStream_t st) {
    if (nr < 1 || nr > 2048 || nf < nr) return set_error(OMB_ERR_INVALID, "row filter: 1 <= rows <= 2048 and Nf >= rows");
    if (ncols <= 0) return OMB_OK;
    const size_t smem = ((size_t)nr * kXS + 2 * (size_t)nr - 1 + kR) * sizeof(float);
    if (cudaFuncSetAttribute(k_circ_filter, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
        return set_error(OMB_ERR_CUDA, "row filter: shared memory attribute failed");
    dim3 block(kCols / kC, (nr + kR - 1) / kR);
    dim3 grid((unsigned)((ncols + kCols - 1) / kCols));
    k_circ_filter<<<grid, block, smem, st>>>(in, out, nr, ncols, L, h, nf, gate);
    OMB_LAUNCH_CHECK("row filter launch");
    return OMB_OK;
}
}  // namespace

int circ_filter(const float *in, float *out, int nr, int64_t ncols, const float *h, int nf, cudaStream_t st) {
    Lines L{1, nr, 0, ncols > 0 ? ncols : 1};
    return launch_lines(in, out, nr, ncols, L, h, nf, FilterGate{}, st);
}

int image_filter(float *g, float *tmp, int nx, int ny, int nz, const float *h, int nf, const FilterGate &gate,
                 cudaStream_t st) {
    if (nx > nf || ny > nf) return set_error(OMB_ERR_INVALID, "image filter: Nf must cover the image's x and y size");
    const int64_t nxy = (int64_t)nx * ny;
    // x lines into tmp, then y lines of tmp back into g (the separable 2-D filter, slice by slice)
    const int64_t nyz = (int64_t)ny * nz;
    Lines Lx{1, nx, 0, nyz};
    int e = launch_lines(g, tmp, nx, nyz, Lx, h, nf, gate, st);
    Lines Ly{nx, 1, nxy, nx};
    if (e == OMB_OK) e = launch_lines(tmp, g, ny, (int64_t)nx * nz, Ly, h, nf, gate, st);
    return e;
}

}  // namespace omb

extern "C" int omb_row_filter(const float *in, float *out, int32_t n_rows, int64_t n_cols, const float *h, int32_t nf,
                              void *stream) {
    if (!in || !out || !h) return omb::set_error(OMB_ERR_INVALID, "NULL pointer passed to omb_row_filter");
    if (in == out) return omb::set_error(OMB_ERR_INVALID, "omb_row_filter: in and out must differ");
    return omb::circ_filter(in, out, n_rows, n_cols, h, nf, (cudaStream_t)stream);
}

extern "C" int omb_image_filter(float *g, float *tmp, int32_t nx, int32_t ny, int32_t nz, const float *h, int32_t nf,
                                void *stream) {
    if (!g || !tmp || !h) return omb::set_error(OMB_ERR_INVALID, "NULL pointer passed to omb_image_filter");
    if (g == tmp) return omb::set_error(OMB_ERR_INVALID, "omb_image_filter: g and tmp must differ");
    if (nx <= 0 || ny <= 0 || nz <= 0) return omb::set_error(OMB_ERR_INVALID, "image size must be positive");
    return omb::image_filter(g, tmp, nx, ny, nz, h, nf, omb::FilterGate{}, (cudaStream_t)stream);
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
