// 3x3x3 convolution of the learned warm start on the 5th-generation tensor
// cores: tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator in tensor
// memory), issued by one thread per CTA.
//
// Implicit GEMM: a CTA computes D[128 voxels][COUT] = sum over 27 taps and
// CIN/16 channel chunks of A[128][16] x B[16][COUT], A the tap-shifted input
// rows (zero outside the volume), B the weights W[tap][co][ci].  Both
// operands are staged in shared memory in the canonical K-major layout
// without swizzle (core matrices of 8 rows x 16 bytes; the two 8-element K
// halves 128 bytes apart, 8-row groups 256 bytes apart), double-buffered: the
// CTA fills stage s^1 while the tensor core reads stage s, and
// tcgen05.commit signals an mbarrier when a stage may be refilled.  The
// epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31 = voxels 32w..), adds the bias, applies the ReLU or the mask
// and stores BF16.  Every mbarrier wait is bounded; on a timeout the CTA
// raises the error flag read by omb_unet_take_error().  The weight gradient
// (k_conv3d_wgrad_tc, below) runs on the same instructions with the voxels
// as the reduction dimension.
#include <cuda_bf16.h>

#include "kernels.h"
#include "../../include/omega_b200_unet.h"

namespace omb {

__device__ int g_unet_error = 0;

namespace tc {

constexpr int kM = 128;              // voxels per CTA (UMMA M)
constexpr int kCoreGroup = 256;      // bytes between 8-row groups (SBO)
constexpr int kKHalf = 128;          // bytes between the two K halves (LBO)
constexpr int kWaitTries = 1 << 20;  // bounded mbarrier polling

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, sm100 (version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((kKHalf >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((kCoreGroup >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;  // base offset 0, LBO mode 0, layout type 0 (no swizzle)
}

// Instruction descriptor: D F32, A/B BF16, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kWaitTries; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc

template <int CIN, int COUT, bool RELU, bool MASK>
__global__ void __launch_bounds__(128) k_conv3d_tc(const __nv_bfloat16 *__restrict__ in,
                                                   const __nv_bfloat16 *__restrict__ w,
                                                   const float *__restrict__ bias, __nv_bfloat16 *__restrict__ out,
                                                   const __nv_bfloat16 *__restrict__ mask, int X, int Y, int Z,
                                                   int64_t nvox) {
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 128, "channel counts");
    constexpr int TMEM_COLS = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : 128);
    constexpr int A_BYTES = tc::kM * 32, B_BYTES = COUT * 32;
    constexpr int KSTEPS = 27 * (CIN / 16);
    __shared__ __align__(1024) uint8_t sA[2][A_BYTES];
    __shared__ __align__(1024) uint8_t sB[2][B_BYTES];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        tc::mbar_init(tc::smem_u32(&bars[0]), 1);
        tc::mbar_init(tc::smem_u32(&bars[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc::smem_u32(&tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;

    // this thread's A row: voxel v (its neighbours change per tap)
    const int64_t v = (int64_t)blockIdx.x * tc::kM + tid;
    const bool vin = v < nvox;
    int x = 0, y = 0, z = 0;
    int64_t b = 0;
    if (vin) {
        int64_t q = v;
        x = (int)(q % X);
        q /= X;
        y = (int)(q % Y);
        q /= Y;
        z = (int)(q % Z);
        b = q / Z;
    }
    const uint32_t idesc = tc::instr_desc(COUT);
    // Step ks uses stage ks & 1; it is that stage's (ks >> 1)-th use, so the
    // commit it waits for before refilling (step ks - 2) completed phase
    // ((ks >> 1) - 1) & 1 of the stage's mbarrier.
    int issued = 0;
    bool ok = true;
    for (int ks = 0; ks < KSTEPS; ++ks) {
        const int tap = ks / (CIN / 16), c = (ks % (CIN / 16)) * 16;
        const int s = ks & 1;
        if (ks >= 2) {
            if (!tc::mbar_wait(tc::smem_u32(&bars[s]), (uint32_t)((ks >> 1) - 1) & 1u)) ok = false;
        }
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        // A row of this thread: 16 channels of the tap-shifted voxel
        {
            const int xs = x + tap % 3 - 1, ys = y + (tap / 3) % 3 - 1, zs = z + tap / 9 - 1;
            uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
            if (vin && xs >= 0 && xs < X && ys >= 0 && ys < Y && zs >= 0 && zs < Z) {
                const uint4 *p = reinterpret_cast<const uint4 *>(in + (((b * Z + zs) * Y + ys) * X + xs) * CIN + c);
                lo = __ldg(p);
                hi = __ldg(p + 1);
            }
            uint8_t *dst = sA[s] + (tid >> 3) * tc::kCoreGroup + (tid & 7) * 16;
            *reinterpret_cast<uint4 *>(dst) = lo;
            *reinterpret_cast<uint4 *>(dst + tc::kKHalf) = hi;
        }
        // B rows: output channel co = tid, 16 input channels
        if (tid < COUT) {
            const uint4 *p = reinterpret_cast<const uint4 *>(w + ((int64_t)tap * COUT + tid) * CIN + c);
            uint8_t *dst = sB[s] + (tid >> 3) * tc::kCoreGroup + (tid & 7) * 16;
            *reinterpret_cast<uint4 *>(dst) = __ldg(p);
            *reinterpret_cast<uint4 *>(dst + tc::kKHalf) = __ldg(p + 1);
        }
        // make the generic-proxy smem writes visible to the tensor core
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            tc::mma_issue(tmem, tc::smem_desc(tc::smem_u32(sA[s])), tc::smem_desc(tc::smem_u32(sB[s])), idesc,
                          ks > 0 ? 1u : 0u);
            tc::mma_commit(tc::smem_u32(&bars[s]));
        }
        issued = ks + 1;
    }
    // the last commit tracks every MMA issued before it
    if (ok) {
        const int last = KSTEPS - 1;
        if (!tc::mbar_wait(tc::smem_u32(&bars[last & 1]), (uint32_t)(last >> 1) & 1u)) ok = false;
    }
    if (!ok) {
        // a commit never arrived: report, give the tensor core a bounded time
        // to finish what it was given, and leave without the epilogue
        if (tid == 0) atomicExch(&g_unet_error, 1);
        if (issued > 0) tc::mbar_wait(tc::smem_u32(&bars[(issued - 1) & 1]), (uint32_t)((issued - 1) >> 1) & 1u);
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (ok) {
        const int64_t vo = (int64_t)blockIdx.x * tc::kM + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float acc[16];
            tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
            if (vo < nvox) {
                __nv_bfloat16 m16[16];
                if (MASK) {
                    const uint4 *mp = reinterpret_cast<const uint4 *>(mask + vo * COUT + c0);
                    *reinterpret_cast<uint4 *>(m16) = __ldg(mp);
                    *reinterpret_cast<uint4 *>(m16 + 8) = __ldg(mp + 1);
                }
                uint32_t packed[8];
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    float lo = acc[i], hi = acc[i + 1];
                    if (bias) {
                        lo += __ldg(bias + c0 + i);
                        hi += __ldg(bias + c0 + i + 1);
                    }
                    if (RELU) {
                        lo = fmaxf(lo, 0.f);
                        hi = fmaxf(hi, 0.f);
                    }
                    if (MASK) {
                        if (!(__bfloat162float(m16[i]) > 0.f)) lo = 0.f;
                        if (!(__bfloat162float(m16[i + 1]) > 0.f)) hi = 0.f;
                    }
                    const __nv_bfloat162 pr = __floats2bfloat162_rn(lo, hi);
                    packed[i / 2] = *reinterpret_cast<const uint32_t *>(&pr);
                }
                uint4 *op = reinterpret_cast<uint4 *>(out + vo * COUT + c0);
                op[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                op[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

#define OMB_TC_SHAPES(X) X(16, 16) X(16, 32) X(32, 32) X(32, 64) X(64, 64) X(96, 32) X(48, 16) \
    X(32, 16) X(64, 32) X(32, 96) X(16, 48)

int unet_conv_tc(int cin, int cout, const void *in, const void *w, const float *bias, void *out, const void *mask,
                 int relu, int X, int Y, int Z, int B, cudaStream_t st) {
    if (X <= 0 || Y <= 0 || Z <= 0 || B <= 0) return set_error(OMB_ERR_INVALID, "bad conv volume");
    const int64_t nvox = (int64_t)X * Y * Z * B;
    const int64_t blocks = (nvox + tc::kM - 1) / tc::kM;
    if (blocks > 2147483647) return set_error(OMB_ERR_UNSUPPORTED, "conv volume too large");
    const auto *i = static_cast<const __nv_bfloat16 *>(in), *wt = static_cast<const __nv_bfloat16 *>(w),
               *mk = static_cast<const __nv_bfloat16 *>(mask);
    auto *o = static_cast<__nv_bfloat16 *>(out);
    const unsigned grid = (unsigned)blocks;
#define X(ci, co)                                                                                   \
    if (cin == ci && cout == co) {                                                                  \
        if (mask)                                                                                   \
            k_conv3d_tc<ci, co, false, true><<<grid, 128, 0, st>>>(i, wt, bias, o, mk, X, Y, Z, nvox);  \
        else if (relu)                                                                              \
            k_conv3d_tc<ci, co, true, false><<<grid, 128, 0, st>>>(i, wt, bias, o, mk, X, Y, Z, nvox);  \
        else                                                                                        \
            k_conv3d_tc<ci, co, false, false><<<grid, 128, 0, st>>>(i, wt, bias, o, mk, X, Y, Z, nvox); \
        OMB_LAUNCH_CHECK("tcgen05 conv launch");                                                    \
        return OMB_OK;                                                                              \
    }
    OMB_TC_SHAPES(X)
#undef X
    return set_error(OMB_ERR_UNSUPPORTED, "conv shape " + std::to_string(cin) + "->" + std::to_string(cout) +
                                              " is not built");
}

// ---------------------------------------------------------------------------
// Weight gradient on the tensor cores.  dW[tap][co][ci] = sum_v dz[v][co]
// in[v + off(tap)][ci] is a GEMM with the voxels as its K dimension:
// D[m][co] = sum_v A[m][v] B[co][v], the rows m = tap * CIN + ci of all 27
// taps taken 128 at a time (grid.y), B = dz.  A CTA reduces `per_cta`
// voxels (grid.x) in stages of 32 (two K = 16 instructions) and adds its
// 128 x COUT partial sums to dW with FP32 atomics.  Both operands are staged
// MN-major (the transpose bits of the instruction descriptor): 8 consecutive
// rows of A are 8 consecutive channels of one tap-shifted input voxel and 8
// consecutive rows of B 8 output channels of one dz voxel, so every 16-byte
// global load lands as one 16-byte row of a core matrix (8 voxels x 16
// bytes).  Core matrix (row group g, voxel group k) lies at g * 256 + k *
// 128 bytes: a row-group stride of 256 (SBO) and a voxel-group stride of 128
// (LBO), the same address map as the K-major operands of the forward kernel,
// so the MMA reads stay inside each 128-row x 16-voxel sub-tile.
// ---------------------------------------------------------------------------
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_conv3d_wgrad_tc(const __nv_bfloat16 *__restrict__ in,
                                                         const __nv_bfloat16 *__restrict__ dz,
                                                         float *__restrict__ dw, int X, int Y, int Z, int64_t nvox,
                                                         int per_cta) {
    static_assert(CIN % 8 == 0 && COUT % 16 == 0 && COUT <= 128, "channel counts");
    constexpr int MROWS = 27 * CIN;
    constexpr int KV = 32;                       // voxels per stage
    constexpr int A_SUB = tc::kM * 16 * 2;       // one K = 16 sub-tile of A (bytes)
    constexpr int B_SUB = COUT * 16 * 2;         // of B
    constexpr int NG = COUT / 8;                 // 8-channel groups of B
    constexpr int TMEM_COLS = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : 128);
    __shared__ __align__(1024) uint8_t sA[2][2 * A_SUB];
    __shared__ __align__(1024) uint8_t sB[2][2 * B_SUB];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base;
    __shared__ short4 vc[2][KV];  // (x, y, z, inside) of each staged voxel
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        tc::mbar_init(tc::smem_u32(&bars[0]), 1);
        tc::mbar_init(tc::smem_u32(&bars[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc::smem_u32(&tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;
    const int m0 = blockIdx.y * tc::kM;
    // this thread's A row group (the same in every stage): tap, first channel and the tap's voxel offset
    const int ga = tid & 15, ma = m0 + ga * 8;
    const bool arow = ma < MROWS;
    const int tapa = arow ? ma / CIN : 0, cia = arow ? ma - tapa * CIN : 0;
    const int ddx = tapa % 3 - 1, ddy = (tapa / 3) % 3 - 1, ddz = tapa / 9 - 1;
    const int64_t doff = ((int64_t)ddz * Y + ddy) * X + ddx;
    const int64_t v_begin = (int64_t)blockIdx.x * per_cta;
    const int64_t v_end = min(v_begin + (int64_t)per_cta, nvox);
    const int nst = (int)((v_end - v_begin + KV - 1) / KV);
    // A and B both MN-major (transpose bits 15 and 16)
    const uint32_t idesc = tc::instr_desc(COUT) | (1u << 15) | (1u << 16);
    // (x, y, z) of voxel v0 + k of a stage, in 32-bit arithmetic (the launch keeps nvox below 2^31)
    auto coords = [&](int st_idx, int buf) {
        if (tid < KV) {
            const int64_t v = v_begin + (int64_t)st_idx * KV + tid;
            short4 c = make_short4(0, 0, 0, 0);
            if (v < v_end) {
                int q = (int)v;
                c.x = (short)(q % X);
                q /= X;
                c.y = (short)(q % Y);
                q /= Y;
                c.z = (short)(q % Z);
                c.w = 1;
            }
            vc[buf][tid] = c;
        }
    };
    int issued = 0;
    bool ok = true;
    if (nst > 0) coords(0, 0);
    for (int ks = 0; ks < nst; ++ks) {
        const int s = ks & 1;
        if (ks >= 2) {
            if (!tc::mbar_wait(tc::smem_u32(&bars[s]), (uint32_t)((ks >> 1) - 1) & 1u)) ok = false;
        }
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        if (ks + 1 < nst) coords(ks + 1, s ^ 1);  // read after the next barrier
        const int64_t v0 = v_begin + (int64_t)ks * KV;
        // A: 32 voxels x 16 row groups, 4 per thread (the voxel k = idx / 16, this thread's row group ga); the
        // voxel coordinates come from the table the previous step filled
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = (tid >> 4) + 8 * j;
            const short4 c = vc[s][k];
            uint4 val = make_uint4(0, 0, 0, 0);
            if (arow && c.w) {
                const int xs = c.x + ddx, ys = c.y + ddy, zs = c.z + ddz;
                if (xs >= 0 && xs < X && ys >= 0 && ys < Y && zs >= 0 && zs < Z)
                    val = __ldg(reinterpret_cast<const uint4 *>(in + (v0 + k + doff) * CIN + cia));
            }
            const int kk = k & 15;
            *reinterpret_cast<uint4 *>(sA[s] + (k >> 4) * A_SUB + ga * tc::kCoreGroup + (kk >> 3) * tc::kKHalf +
                                       (kk & 7) * 16) = val;
        }
        // B: 32 voxels x NG channel groups
        for (int idx = tid; idx < KV * NG; idx += 128) {
            const int k = idx / NG, g = idx - k * NG;
            const int64_t v = v0 + k;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (v < v_end) val = __ldg(reinterpret_cast<const uint4 *>(dz + v * COUT + g * 8));
            const int kk = k & 15;
            *reinterpret_cast<uint4 *>(sB[s] + (k >> 4) * B_SUB + g * tc::kCoreGroup + (kk >> 3) * tc::kKHalf +
                                       (kk & 7) * 16) = val;
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
            for (int sub = 0; sub < 2; ++sub)
                tc::mma_issue(tmem, tc::smem_desc(tc::smem_u32(sA[s] + sub * A_SUB)),
                              tc::smem_desc(tc::smem_u32(sB[s] + sub * B_SUB)), idesc, (ks > 0 || sub > 0) ? 1u : 0u);
            tc::mma_commit(tc::smem_u32(&bars[s]));
        }
        issued = ks + 1;
    }
    if (ok && nst > 0) {
        const int last = nst - 1;
        if (!tc::mbar_wait(tc::smem_u32(&bars[last & 1]), (uint32_t)(last >> 1) & 1u)) ok = false;
    }
    if (!ok) {
        if (tid == 0) atomicExch(&g_unet_error, 1);
        if (issued > 0) tc::mbar_wait(tc::smem_u32(&bars[(issued - 1) & 1]), (uint32_t)((issued - 1) >> 1) & 1u);
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (ok && nst > 0) {
        // row m of D = TMEM lane m: warp w holds rows 32w..32w+31
        const int m = m0 + warp * 32 + lane;
        const bool mrow = m < MROWS;
        const int tap = mrow ? m / CIN : 0, ci = mrow ? m - tap * CIN : 0;
        float *d = dw + (int64_t)tap * COUT * CIN + ci;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float acc[16];
            tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
            if (mrow) {
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(d + (c0 + i) * CIN, acc[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

int unet_conv_wgrad_tc(int cin, int cout, const void *in, const void *dz, float *dw, int X, int Y, int Z, int B,
                       cudaStream_t st) {
    if (X <= 0 || Y <= 0 || Z <= 0 || B <= 0) return set_error(OMB_ERR_INVALID, "bad conv volume");
    const int64_t nvox = (int64_t)X * Y * Z * B;
    const int per_cta = 32 * 256;  // voxels per CTA (a multiple of the 32-voxel stage)
    const int64_t chunks = (nvox + per_cta - 1) / per_cta;
    if (nvox > 2147483647 || X > 32767 || Y > 32767 || Z > 32767)
        return set_error(OMB_ERR_UNSUPPORTED, "wgrad volume too large (2^31 voxels, 32767 per axis)");
    const auto *i = static_cast<const __nv_bfloat16 *>(in), *d = static_cast<const __nv_bfloat16 *>(dz);
#define X(ci, co)                                                                                             \
    if (cin == ci && cout == co) {                                                                            \
        dim3 grid((unsigned)chunks, (unsigned)((27 * ci + tc::kM - 1) / tc::kM));                              \
        k_conv3d_wgrad_tc<ci, co><<<grid, 128, 0, st>>>(i, d, dw, X, Y, Z, nvox, per_cta);                     \
        OMB_LAUNCH_CHECK("tcgen05 wgrad launch");                                                             \
        return OMB_OK;                                                                                        \
    }
    OMB_TC_SHAPES(X)
#undef X
    return set_error(OMB_ERR_UNSUPPORTED, "wgrad shape " + std::to_string(cin) + "->" + std::to_string(cout) +
                                              " is not built");
}

}  // namespace omb

extern "C" {

int omb_unet_conv_tc(int32_t cin, int32_t cout, const void *in, const void *w, const float *bias, void *out,
                     const void *relu_mask, int32_t relu, int32_t X, int32_t Y, int32_t Z, int32_t B, void *stream) {
    if (!in || !w || !out) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_conv_tc");
    return omb::unet_conv_tc(cin, cout, in, w, bias, out, relu_mask, relu, X, Y, Z, B, (cudaStream_t)stream);
}

int omb_unet_conv_wgrad_tc(int32_t cin, int32_t cout, const void *in, const void *dz, float *dw, int32_t X,
                           int32_t Y, int32_t Z, int32_t B, void *stream) {
    if (!in || !dz || !dw) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_conv_wgrad_tc");
    return omb::unet_conv_wgrad_tc(cin, cout, in, dz, dw, X, Y, Z, B, (cudaStream_t)stream);
}

int omb_unet_take_error(int32_t *out_host) {
    if (!out_host) return omb::set_error(OMB_ERR_INVALID, "output pointer is NULL");
    int v = 0;
    const cudaError_t e = cudaMemcpyFromSymbol(&v, omb::g_unet_error, sizeof(int));
    if (e != cudaSuccess) return omb::cuda_fail(e, "read conv error flag");
    const int zero = 0;
    const cudaError_t e2 = cudaMemcpyToSymbol(omb::g_unet_error, &zero, sizeof(int));
    if (e2 != cudaSuccess) return omb::cuda_fail(e2, "clear conv error flag");
    *out_host = v;
    return OMB_OK;
}

}  // extern "C"
