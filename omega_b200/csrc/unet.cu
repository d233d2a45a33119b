// Kernels of the learned OSEM warm start: a small 3-D U-Net (3x3x3
// convolutions, BF16 weights and activations, FP32 accumulation) trained and
// run on the GPU by these kernels alone.
//
// Layouts: activations are channels-last BF16, [B][Z][Y][X][C] with C a
// multiple of 16; conv weights are BF16 [27][Cout][Cin] (tap-major, input
// channels contiguous), tap = (dz+1)*9 + (dy+1)*3 + (dx+1); biases FP32.
//
// Convolutions are implicit GEMMs on the tensor cores (mma.sync m16n8k16,
// BF16 in, FP32 accumulate):
//   forward  out[v][co] = relu(bias[co] + sum_tap sum_ci in[v+off(tap)][ci] W[tap][co][ci])
//   dgrad    the same kernel on the flipped, transposed weights
//            W'[tap][ci][co] = W[26 - tap][co][ci] (off(26 - tap) = -off(tap)),
//            with the next ReLU's derivative fused as a mask on the output
//   wgrad    dW[tap][co][ci] = sum_v dz[v][co] in[v+off(tap)][ci]: voxels are
//            the GEMM's K; tiles of 128 voxels staged in shared memory and read
//            transposed with ldmatrix.trans, partial sums added with FP32 atomics.
#include <cuda_bf16.h>

#include "kernels.h"
#include "../../include/omega_b200_unet.h"

namespace omb {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld_pair(const bf16 *p) { return __ldg(reinterpret_cast<const unsigned int *>(p)); }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// ---------------------------------------------------------------------------
// Forward / dgrad convolution.  Block = 4 warps = 64 consecutive voxels along
// x of one (y, z, batch) row; warp = 16 voxels x COUT channels.
// ---------------------------------------------------------------------------
template <int CIN, int COUT, bool RELU, bool MASK>
__global__ void __launch_bounds__(128) k_conv3d(const bf16 *__restrict__ in, const bf16 *__restrict__ w,
                                                const float *__restrict__ bias, bf16 *__restrict__ out,
                                                const bf16 *__restrict__ mask, int X, int Y, int Z) {
    static_assert(CIN % 16 == 0 && COUT % 8 == 0, "channel counts");
    constexpr int NT = COUT / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int y = blockIdx.y;
    const int z = blockIdx.z % Z, b = blockIdx.z / Z;
    const int xbase = blockIdx.x * 64 + warp * 16;
    const int xr0 = xbase + g, xr1 = xbase + g + 8;  // the two A rows of this thread
    const int64_t row_off = (((int64_t)b * Z + z) * Y + y) * X;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    if (xbase < X) {
        for (int tap = 0; tap < 27; ++tap) {
            const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
            const int zz = z + dz, yy = y + dy;
            if (zz < 0 || zz >= Z || yy < 0 || yy >= Y) continue;
            const int x0 = xr0 + dx, x1 = xr1 + dx;
            const bool v0 = x0 >= 0 && x0 < X, v1 = x1 >= 0 && x1 < X;
            const int64_t base = (((int64_t)b * Z + zz) * Y + yy) * X;
            const bf16 *p0 = in + (base + (v0 ? x0 : 0)) * CIN + 2 * t;
            const bf16 *p1 = in + (base + (v1 ? x1 : 0)) * CIN + 2 * t;
            const bf16 *wt = w + (int64_t)tap * COUT * CIN + (int64_t)g * CIN + 2 * t;
#pragma unroll
            for (int c = 0; c < CIN; c += 16) {
                const uint32_t a0 = v0 ? ld_pair(p0 + c) : 0u, a1 = v1 ? ld_pair(p1 + c) : 0u;
                const uint32_t a2 = v0 ? ld_pair(p0 + c + 8) : 0u, a3 = v1 ? ld_pair(p1 + c + 8) : 0u;
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    const bf16 *wj = wt + (int64_t)j * 8 * CIN + c;
                    mma_bf16(acc[j], a0, a1, a2, a3, ld_pair(wj), ld_pair(wj + 8));
                }
            }
        }
    }
    // epilogue: rows g and g+8, channels j*8 + 2t, +1
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int xr = h ? xr1 : xr0;
        if (xr >= X) continue;
        const int64_t v = row_off + xr;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int co = j * 8 + 2 * t;
            float lo = acc[j][2 * h], hi = acc[j][2 * h + 1];
            if (bias) {
                lo += __ldg(bias + co);
                hi += __ldg(bias + co + 1);
            }
            if (RELU) {
                lo = fmaxf(lo, 0.f);
                hi = fmaxf(hi, 0.f);
            }
            if (MASK) {
                const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162 *>(mask + v * COUT + co);
                if (!(__low2float(m) > 0.f)) lo = 0.f;
                if (!(__high2float(m) > 0.f)) hi = 0.f;
            }
            *reinterpret_cast<uint32_t *>(out + v * COUT + co) = pack_bf16(lo, hi);
        }
    }
}

// ---------------------------------------------------------------------------
// Weight gradient.  grid = (chunks, 27); block = 4 warps; each block reduces
// `per_block` voxels (multiple of 128) for one tap.
// ---------------------------------------------------------------------------
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_conv3d_wgrad(const bf16 *__restrict__ in, const bf16 *__restrict__ dz,
                                                      float *__restrict__ dw, int X, int Y, int Z, int64_t nvox,
                                                      int per_block) {
    constexpr int SA = COUT + 8, SB = CIN + 8;  // padded smem rows (bank spread for ldmatrix)
    __shared__ __align__(16) bf16 sA[128 * SA];
    __shared__ __align__(16) bf16 sB[128 * SB];
    constexpr int MT = COUT / 16, NT = CIN / 8, TILES = MT * NT;
    constexpr int PER_WARP = (TILES + 3) / 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tap = blockIdx.y;
    const int ddz = tap / 9 - 1, ddy = (tap / 3) % 3 - 1, ddx = tap % 3 - 1;
    float acc[PER_WARP][4];
#pragma unroll
    for (int i = 0; i < PER_WARP; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    const int64_t v_begin = (int64_t)blockIdx.x * per_block;
    const int64_t v_end = min(v_begin + (int64_t)per_block, nvox);
    for (int64_t v0 = v_begin; v0 < v_end; v0 += 128) {
        // stage: thread r loads voxel v0 + r's dz row and its tap-shifted input row
        {
            const int r = threadIdx.x;
            const int64_t v = v0 + r;
            bool ok = v < v_end;
            int64_t src = 0;
            if (ok) {
                const int x = (int)(v % X);
                const int64_t q = v / X;
                const int yv = (int)(q % Y);
                const int64_t q2 = q / Y;
                const int zv = (int)(q2 % Z);
                const int64_t bb = q2 / Z;
                const int xs = x + ddx, ys = yv + ddy, zs = zv + ddz;
                if (xs >= 0 && xs < X && ys >= 0 && ys < Y && zs >= 0 && zs < Z)
                    src = ((bb * Z + zs) * Y + ys) * X + xs;
                else
                    src = -1;
            }
            const uint4 zero4 = make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int c = 0; c < COUT; c += 8)
                *reinterpret_cast<uint4 *>(sA + r * SA + c) =
                    ok ? __ldg(reinterpret_cast<const uint4 *>(dz + v * COUT + c)) : zero4;
#pragma unroll
            for (int c = 0; c < CIN; c += 8)
                *reinterpret_cast<uint4 *>(sB + r * SB + c) =
                    (ok && src >= 0) ? __ldg(reinterpret_cast<const uint4 *>(in + src * CIN + c)) : zero4;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 128; k += 16) {
#pragma unroll
            for (int i = 0; i < PER_WARP; ++i) {
                const int tile = warp + 4 * i;
                if (tile < TILES) {
                    const int mt = tile / NT, nt = tile % NT;
                    // A = dz^T (co x voxel): ldmatrix.x4.trans of sA rows k.., columns mt*16..
                    const int mi = lane >> 3, rr = lane & 7;
                    const bf16 *pa = sA + (k + rr + (mi >> 1) * 8) * SA + mt * 16 + (mi & 1) * 8;
                    uint32_t a0, a1, a2, a3;
                    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(pa);
                    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                                 : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
                                 : "r"(sa));
                    // B = input (voxel x ci): ldmatrix.x2.trans of sB rows k.., columns nt*8..
                    const int mb = (lane >> 3) & 1;
                    const bf16 *pb = sB + (k + rr + mb * 8) * SB + nt * 8;
                    uint32_t b0, b1;
                    const uint32_t sb = (uint32_t)__cvta_generic_to_shared(pb);
                    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                                 : "=r"(b0), "=r"(b1)
                                 : "r"(sb));
                    mma_bf16(acc[i], a0, a1, a2, a3, b0, b1);
                }
            }
        }
        __syncthreads();
    }
    // D fragment: rows (co) mt*16 + g (+8), columns (ci) nt*8 + 2t (+1)
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int i = 0; i < PER_WARP; ++i) {
        const int tile = warp + 4 * i;
        if (tile < TILES) {
            const int mt = tile / NT, nt = tile % NT;
            float *d = dw + (int64_t)tap * COUT * CIN;
            const int co = mt * 16 + g, ci = nt * 8 + 2 * t;
            atomicAdd(d + co * CIN + ci, acc[i][0]);
            atomicAdd(d + co * CIN + ci + 1, acc[i][1]);
            atomicAdd(d + (co + 8) * CIN + ci, acc[i][2]);
            atomicAdd(d + (co + 8) * CIN + ci + 1, acc[i][3]);
        }
    }
}

// Bias gradient: db[co] = sum_v dz[v][co] (FP32 atomics per block).
template <int C>
__global__ void k_bias_grad(const bf16 *__restrict__ dz, float *__restrict__ db, int64_t nvox) {
    __shared__ float part[C];
    for (int c = threadIdx.x; c < C; c += blockDim.x) part[c] = 0.f;
    __syncthreads();
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    float s = 0.f;
    for (int64_t v = (int64_t)blockIdx.x * lanes + threadIdx.x / C; v < nvox; v += (int64_t)gridDim.x * lanes)
        s += __bfloat162float(dz[v * C + c]);
    atomicAdd(part + c, s);
    __syncthreads();
    for (int cc = threadIdx.x; cc < C; cc += blockDim.x) atomicAdd(db + cc, part[cc]);
}

// d = d * (a > 0) in place (the derivative of a = relu(z) applied to dL/da).
__global__ void k_relu_mask(bf16 *__restrict__ d, const bf16 *__restrict__ a, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!(__bfloat162float(a[i]) > 0.f)) d[i] = __float2bfloat16(0.f);
}

// W'[tap][ci][co] = W[26 - tap][co][ci]
__global__ void k_flip_weights(const bf16 *__restrict__ w, bf16 *__restrict__ wf, int cin, int cout) {
    const int n = 27 * cin * cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int tap = i / (cin * cout), r = i % (cin * cout);
        const int ci = r / cout, co = r % cout;
        wf[i] = w[(int64_t)(26 - tap) * cout * cin + (int64_t)co * cin + ci];
    }
}

// ---------------------------------------------------------------------------
// Resampling and channel plumbing (channels-last BF16)
// ---------------------------------------------------------------------------

// 2x2x2 average pooling: out [B][Z/2][Y/2][X/2][C].
__global__ void k_avgpool2(const bf16 *__restrict__ in, bf16 *__restrict__ out, int X, int Y, int Z, int C,
                           int64_t nout) {
    const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nout * C; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        int64_t v = i / C;
        const int x = (int)(v % Xo);
        v /= Xo;
        const int y = (int)(v % Yo);
        v /= Yo;
        const int z = (int)(v % Zo);
        const int64_t b = v / Zo;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int xx = 2 * x + (k & 1), yy = 2 * y + ((k >> 1) & 1), zz = 2 * z + (k >> 2);
            s += __bfloat162float(in[((((b * Z) + zz) * Y + yy) * X + xx) * C + c]);
        }
        out[i] = __float2bfloat16(0.125f * s);
    }
}

// Backward of the average pooling, accumulated: din[child] += dout[parent] / 8.
__global__ void k_avgpool2_bwd(const bf16 *__restrict__ dout, bf16 *__restrict__ din, int X, int Y, int Z, int C,
                               int64_t nin) {
    const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nin * C; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        int64_t v = i / C;
        const int x = (int)(v % X);
        v /= X;
        const int y = (int)(v % Y);
        v /= Y;
        const int z = (int)(v % Z);
        const int64_t b = v / Z;
        const int64_t p = (((b * Zo + z / 2) * Yo + y / 2) * Xo + x / 2) * C + c;
        din[i] = __float2bfloat16(__bfloat162float(din[i]) + 0.125f * __bfloat162float(dout[p]));
    }
}

// Nearest 2x upsampling of `low` ([B][Z/2][Y/2][X/2][Cl]) written into channels
// [0, Cl) of `cat` ([B][Z][Y][X][Cl + Cs]) and `skip` ([..][Cs]) into [Cl, Cl + Cs).
__global__ void k_up_concat(const bf16 *__restrict__ low, const bf16 *__restrict__ skip, bf16 *__restrict__ cat,
                            int X, int Y, int Z, int Cl, int Cs, int64_t nvox) {
    const int C = Cl + Cs;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvox * C; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const int64_t v = i / C;
        if (c >= Cl) {
            cat[i] = skip[v * Cs + (c - Cl)];
        } else {
            int64_t q = v;
            const int x = (int)(q % X);
            q /= X;
            const int y = (int)(q % Y);
            q /= Y;
            const int z = (int)(q % Z);
            const int64_t b = q / Z;
            cat[i] = low[(((b * (Z / 2) + z / 2) * (Y / 2) + y / 2) * (X / 2) + x / 2) * Cl + c];
        }
    }
}

// Backward of k_up_concat: dlow[parent] = sum of the 8 children's first Cl
// channels; dskip += the remaining Cs channels (added to the gradient that
// already flows into the skip tensor).
__global__ void k_up_concat_bwd(const bf16 *__restrict__ dcat, bf16 *__restrict__ dlow, bf16 *__restrict__ dskip,
                                int X, int Y, int Z, int Cl, int Cs, int64_t nlow, int64_t nvox) {
    const int C = Cl + Cs;
    const int Xl = X / 2, Yl = Y / 2, Zl = Z / 2;
    const int64_t total_low = nlow * Cl, total_skip = nvox * Cs;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total_low + total_skip;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < total_low) {
            const int c = (int)(i % Cl);
            int64_t q = i / Cl;
            const int x = (int)(q % Xl);
            q /= Xl;
            const int y = (int)(q % Yl);
            q /= Yl;
            const int z = (int)(q % Zl);
            const int64_t b = q / Zl;
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int xx = 2 * x + (k & 1), yy = 2 * y + ((k >> 1) & 1), zz = 2 * z + (k >> 2);
                s += __bfloat162float(dcat[((((b * Z) + zz) * Y + yy) * X + xx) * C + c]);
            }
            dlow[i] = __float2bfloat16(s);
        } else {
            const int64_t j = i - total_low;
            const int c = (int)(j % Cs);
            const int64_t v = j / Cs;
            dskip[j] = __float2bfloat16(__bfloat162float(dskip[j]) + __bfloat162float(dcat[v * C + Cl + c]));
        }
    }
}

// ---------------------------------------------------------------------------
// Network input / output
// ---------------------------------------------------------------------------

// Input tensor [B][Z][Y][X][16] from the Fortran-order FP32 volumes: channel 0
// = osem[b] * scale[b], channel 1 = sens * sens_scale, other channels 0.
// Source volumes have Zs <= Z slices (the rest is zero padding).
__global__ void k_make_input(const float *__restrict__ osem, int64_t osem_stride, const float *__restrict__ sens,
                             const float *__restrict__ scale, float sens_scale, bf16 *__restrict__ out, int X, int Y,
                             int Z, int Zs, int64_t nvox) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t q = v;
        const int x = (int)(q % X);
        q /= X;
        const int y = (int)(q % Y);
        q /= Y;
        const int z = (int)(q % Z);
        const int64_t b = q / Z;
        float c0 = 0.f, c1 = 0.f;
        if (z < Zs) {
            const int64_t s = x + (int64_t)X * (y + (int64_t)Y * z);
            c0 = osem[b * osem_stride + s] * scale[b];
            c1 = sens[s] * sens_scale;
        }
        uint4 *o = reinterpret_cast<uint4 *>(out + v * 16);
        o[0] = make_uint4(pack_bf16(c0, c1), 0u, 0u, 0u);
        o[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Head: pred[b][v] = osem_n[b][v] + bias + sum_c w[c] a[v][c] (a: [..][16]),
// written as FP32 in the padded volume order.
__global__ void k_head_fwd(const bf16 *__restrict__ a, const bf16 *__restrict__ inp, const float *__restrict__ w,
                           const float *__restrict__ bias, float *__restrict__ pred, int64_t nvox) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
        float s = __bfloat162float(inp[v * 16]) + bias[0];
#pragma unroll
        for (int c = 0; c < 16; ++c) s = fmaf(w[c], __bfloat162float(a[v * 16 + c]), s);
        pred[v] = s;
    }
}

// Loss and head backward: r = pred - target on the valid slices (z < Zs),
// loss += sum r^2 / count; d a[v][c] = g w[c] masked by relu(a) > 0, g = 2 r / count;
// dw[c] += g a[v][c]; db += g.
__global__ void k_head_bwd(const bf16 *__restrict__ a, const float *__restrict__ pred,
                           const float *__restrict__ target, int64_t target_stride, const float *__restrict__ tscale,
                           const float *__restrict__ w, bf16 *__restrict__ da, float *__restrict__ dw,
                           float *__restrict__ db, float *__restrict__ loss, int X, int Y, int Z, int Zs,
                           int64_t nvox, float inv_count) {
    __shared__ float sw[17];
    __shared__ float sl;
    if (threadIdx.x < 17) sw[threadIdx.x] = 0.f;
    if (threadIdx.x == 0) sl = 0.f;
    __syncthreads();
    float lw[16], lb = 0.f, ll = 0.f;
#pragma unroll
    for (int c = 0; c < 16; ++c) lw[c] = 0.f;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t q = v;
        const int x = (int)(q % X);
        q /= X;
        const int y = (int)(q % Y);
        q /= Y;
        const int z = (int)(q % Z);
        const int64_t b = q / Z;
        float gr = 0.f;
        if (z < Zs) {
            const float tv = target[b * target_stride + x + (int64_t)X * (y + (int64_t)Y * z)] * tscale[b];
            const float r = pred[v] - tv;
            ll = fmaf(r, r, ll);
            gr = 2.f * r * inv_count;
        }
        lb += gr;
#pragma unroll
        for (int c = 0; c < 16; c += 2) {
            const float a0 = __bfloat162float(a[v * 16 + c]), a1 = __bfloat162float(a[v * 16 + c + 1]);
            lw[c] = fmaf(gr, a0, lw[c]);
            lw[c + 1] = fmaf(gr, a1, lw[c + 1]);
            const float d0 = a0 > 0.f ? gr * w[c] : 0.f, d1 = a1 > 0.f ? gr * w[c + 1] : 0.f;
            *reinterpret_cast<uint32_t *>(da + v * 16 + c) = pack_bf16(d0, d1);
        }
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) atomicAdd(sw + c, lw[c]);
    atomicAdd(sw + 16, lb);
    atomicAdd(&sl, ll * inv_count);
    __syncthreads();
    if (threadIdx.x < 16) atomicAdd(dw + threadIdx.x, sw[threadIdx.x]);
    if (threadIdx.x == 16) atomicAdd(db, sw[16]);
    if (threadIdx.x == 0) atomicAdd(loss, sl);
}

// Network output back to Fortran-order FP32 volumes: out[b][s] = pred / scale[b], clamped >= floor.
__global__ void k_head_out(const float *__restrict__ pred, const float *__restrict__ scale, float *__restrict__ out,
                           int64_t out_stride, float floor_v, int X, int Y, int Z, int Zs, int64_t nvox) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t q = v;
        const int x = (int)(q % X);
        q /= X;
        const int y = (int)(q % Y);
        q /= Y;
        const int z = (int)(q % Z);
        const int64_t b = q / Z;
        if (z < Zs) out[b * out_stride + x + (int64_t)X * (y + (int64_t)Y * z)] = fmaxf(pred[v] / scale[b], floor_v);
    }
}

// Adam on FP32 master weights; writes the BF16 copy used by the kernels.
__global__ void k_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ gr, bf16 *__restrict__ pb, int64_t n, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float g = gr[i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float upd = lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] -= upd;
        if (pb) pb[i] = __float2bfloat16(p[i]);
    }
}

__global__ void k_f32_to_bf16(const float *__restrict__ a, bf16 *__restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16(a[i]);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

#define OMB_CONV_SHAPES(X) X(16, 16) X(16, 32) X(32, 32) X(32, 64) X(64, 64) X(96, 32) X(48, 16) \
    X(32, 16) X(64, 32) X(32, 96) X(16, 48)

int unet_conv(int cin, int cout, const void *in, const void *w, const float *bias, void *out, const void *mask,
              int relu, int X, int Y, int Z, int B, cudaStream_t st) {
    if (X <= 0 || Y <= 0 || Z <= 0 || B <= 0) return set_error(OMB_ERR_INVALID, "bad conv volume");
    if ((int64_t)Z * B > 65535 || Y > 65535) return set_error(OMB_ERR_UNSUPPORTED, "conv volume too large");
    dim3 grid((X + 63) / 64, Y, Z * B);
    const bf16 *i = static_cast<const bf16 *>(in), *wt = static_cast<const bf16 *>(w),
               *mk = static_cast<const bf16 *>(mask);
    bf16 *o = static_cast<bf16 *>(out);
#define X(ci, co)                                                                                   \
    if (cin == ci && cout == co) {                                                                  \
        if (mask)                                                                                   \
            k_conv3d<ci, co, false, true><<<grid, 128, 0, st>>>(i, wt, bias, o, mk, X, Y, Z);       \
        else if (relu)                                                                              \
            k_conv3d<ci, co, true, false><<<grid, 128, 0, st>>>(i, wt, bias, o, mk, X, Y, Z);       \
        else                                                                                        \
            k_conv3d<ci, co, false, false><<<grid, 128, 0, st>>>(i, wt, bias, o, mk, X, Y, Z);      \
        OMB_LAUNCH_CHECK("conv launch");                                                            \
        return OMB_OK;                                                                              \
    }
    OMB_CONV_SHAPES(X)
#undef X
    return set_error(OMB_ERR_UNSUPPORTED, "conv shape " + std::to_string(cin) + "->" + std::to_string(cout) +
                                              " is not built");
}

int unet_conv_wgrad(int cin, int cout, const void *in, const void *dz, float *dw, int X, int Y, int Z, int B,
                    cudaStream_t st) {
    const int64_t nvox = (int64_t)X * Y * Z * B;
    const int per_block = 128 * 64;
    const int64_t chunks = (nvox + per_block - 1) / per_block;
    if (chunks > 2147483647) return set_error(OMB_ERR_UNSUPPORTED, "wgrad volume too large");
    dim3 grid((unsigned)chunks, 27);
    const bf16 *i = static_cast<const bf16 *>(in), *d = static_cast<const bf16 *>(dz);
#define X(ci, co)                                                                                          \
    if (cin == ci && cout == co) {                                                                         \
        k_conv3d_wgrad<ci, co><<<grid, 128, 0, st>>>(i, d, dw, X, Y, Z, nvox, per_block);                  \
        OMB_LAUNCH_CHECK("wgrad launch");                                                                  \
        return OMB_OK;                                                                                     \
    }
    OMB_CONV_SHAPES(X)
#undef X
    return set_error(OMB_ERR_UNSUPPORTED, "wgrad shape is not built");
}

int unet_bias_grad(int c, const void *dz, float *db, int64_t nvox, cudaStream_t st) {
    const bf16 *d = static_cast<const bf16 *>(dz);
    const unsigned grid = grid_for(nvox * c / 256 + 1, 4);
    switch (c) {
        case 16: k_bias_grad<16><<<grid, 256, 0, st>>>(d, db, nvox); break;
        case 32: k_bias_grad<32><<<grid, 256, 0, st>>>(d, db, nvox); break;
        case 64: k_bias_grad<64><<<grid, 256, 0, st>>>(d, db, nvox); break;
        default: return set_error(OMB_ERR_UNSUPPORTED, "bias gradient channel count");
    }
    OMB_LAUNCH_CHECK("bias grad launch");
    return OMB_OK;
}

int unet_flip_weights(const void *w, void *wf, int cin, int cout, cudaStream_t st) {
    k_flip_weights<<<grid_for(27 * cin * cout, 2), 256, 0, st>>>(static_cast<const bf16 *>(w), static_cast<bf16 *>(wf),
                                                                 cin, cout);
    OMB_LAUNCH_CHECK("flip launch");
    return OMB_OK;
}

int unet_avgpool(const void *in, void *out, int X, int Y, int Z, int B, int C, int backward, cudaStream_t st) {
    if (X % 2 || Y % 2 || Z % 2) return set_error(OMB_ERR_INVALID, "pooling needs even sizes");
    if (!backward) {
        const int64_t nout = (int64_t)(X / 2) * (Y / 2) * (Z / 2) * B;
        k_avgpool2<<<grid_for(nout * C, 8), 256, 0, st>>>(static_cast<const bf16 *>(in), static_cast<bf16 *>(out), X,
                                                          Y, Z, C, nout);
    } else {
        const int64_t nin = (int64_t)X * Y * Z * B;
        k_avgpool2_bwd<<<grid_for(nin * C, 8), 256, 0, st>>>(static_cast<const bf16 *>(in), static_cast<bf16 *>(out),
                                                             X, Y, Z, C, nin);
    }
    OMB_LAUNCH_CHECK("pool launch");
    return OMB_OK;
}

int unet_up_concat(const void *low, const void *skip, void *cat, int X, int Y, int Z, int B, int cl, int cs,
                   cudaStream_t st) {
    const int64_t nvox = (int64_t)X * Y * Z * B;
    k_up_concat<<<grid_for(nvox * (cl + cs), 8), 256, 0, st>>>(static_cast<const bf16 *>(low),
                                                               static_cast<const bf16 *>(skip), static_cast<bf16 *>(cat),
                                                               X, Y, Z, cl, cs, nvox);
    OMB_LAUNCH_CHECK("upsample launch");
    return OMB_OK;
}

int unet_up_concat_bwd(const void *dcat, void *dlow, void *dskip, int X, int Y, int Z, int B, int cl, int cs,
                       cudaStream_t st) {
    const int64_t nvox = (int64_t)X * Y * Z * B, nlow = nvox / 8;
    k_up_concat_bwd<<<grid_for(nlow * cl + nvox * cs, 8), 256, 0, st>>>(
        static_cast<const bf16 *>(dcat), static_cast<bf16 *>(dlow), static_cast<bf16 *>(dskip), X, Y, Z, cl, cs, nlow,
        nvox);
    OMB_LAUNCH_CHECK("upsample backward launch");
    return OMB_OK;
}

int unet_make_input(const float *osem, int64_t osem_stride, const float *sens, const float *scale, float sens_scale,
                    void *out, int X, int Y, int Z, int Zs, int B, cudaStream_t st) {
    const int64_t nvox = (int64_t)X * Y * Z * B;
    k_make_input<<<grid_for(nvox, 8), 256, 0, st>>>(osem, osem_stride, sens, scale, sens_scale,
                                                    static_cast<bf16 *>(out), X, Y, Z, Zs, nvox);
    OMB_LAUNCH_CHECK("input launch");
    return OMB_OK;
}

int unet_head_fwd(const void *a, const void *inp, const float *w, const float *bias, float *pred, int64_t nvox,
                  cudaStream_t st) {
    k_head_fwd<<<grid_for(nvox, 8), 256, 0, st>>>(static_cast<const bf16 *>(a), static_cast<const bf16 *>(inp), w,
                                                  bias, pred, nvox);
    OMB_LAUNCH_CHECK("head launch");
    return OMB_OK;
}

int unet_head_bwd(const void *a, const float *pred, const float *target, int64_t target_stride, const float *tscale,
                  const float *w, void *da, float *dw, float *db, float *loss, int X, int Y, int Z, int Zs, int B,
                  cudaStream_t st) {
    const int64_t nvox = (int64_t)X * Y * Z * B;
    const float inv = 1.f / (float)((int64_t)X * Y * Zs * B);
    k_head_bwd<<<grid_for(nvox, 4), 256, 0, st>>>(static_cast<const bf16 *>(a), pred, target, target_stride, tscale, w,
                                                  static_cast<bf16 *>(da), dw, db, loss, X, Y, Z, Zs, nvox, inv);
    OMB_LAUNCH_CHECK("head backward launch");
    return OMB_OK;
}

int unet_head_out(const float *pred, const float *scale, float *out, int64_t out_stride, float floor_v, int X, int Y,
                  int Z, int Zs, int B, cudaStream_t st) {
    const int64_t nvox = (int64_t)X * Y * Z * B;
    k_head_out<<<grid_for(nvox, 8), 256, 0, st>>>(pred, scale, out, out_stride, floor_v, X, Y, Z, Zs, nvox);
    OMB_LAUNCH_CHECK("output launch");
    return OMB_OK;
}

int unet_adam(float *p, float *m, float *v, const float *g, void *pb, int64_t n, float lr, float b1, float b2,
              int step, float eps, cudaStream_t st) {
    const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
    k_adam<<<grid_for(n, 4), 256, 0, st>>>(p, m, v, g, static_cast<bf16 *>(pb), n, lr, b1, b2, c1, c2, eps);
    OMB_LAUNCH_CHECK("adam launch");
    return OMB_OK;
}

int unet_relu_mask(void *d, const void *a, int64_t n, cudaStream_t st) {
    k_relu_mask<<<grid_for(n, 8), 256, 0, st>>>(static_cast<bf16 *>(d), static_cast<const bf16 *>(a), n);
    OMB_LAUNCH_CHECK("relu mask launch");
    return OMB_OK;
}

int unet_to_bf16(const float *a, void *b, int64_t n, cudaStream_t st) {
    k_f32_to_bf16<<<grid_for(n, 4), 256, 0, st>>>(a, static_cast<bf16 *>(b), n);
    OMB_LAUNCH_CHECK("bf16 conversion launch");
    return OMB_OK;
}

}  // namespace omb

// ---------------------------------------------------------------------------
// C-ABI (include/omega_b200_unet.h)
// ---------------------------------------------------------------------------
extern "C" {

int omb_unet_conv(int32_t cin, int32_t cout, const void *in, const void *w, const float *bias, void *out,
                  const void *relu_mask, int32_t relu, int32_t X, int32_t Y, int32_t Z, int32_t B, void *stream) {
    if (!in || !w || !out) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_conv");
    return omb::unet_conv(cin, cout, in, w, bias, out, relu_mask, relu, X, Y, Z, B, (cudaStream_t)stream);
}

int omb_unet_conv_wgrad(int32_t cin, int32_t cout, const void *in, const void *dz, float *dw, int32_t X, int32_t Y,
                        int32_t Z, int32_t B, void *stream) {
    if (!in || !dz || !dw) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_conv_wgrad");
    return omb::unet_conv_wgrad(cin, cout, in, dz, dw, X, Y, Z, B, (cudaStream_t)stream);
}

int omb_unet_bias_grad(int32_t c, const void *dz, float *db, int64_t nvox, void *stream) {
    if (!dz || !db) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_bias_grad");
    return omb::unet_bias_grad(c, dz, db, nvox, (cudaStream_t)stream);
}

int omb_unet_flip_weights(const void *w, void *wf, int32_t cin, int32_t cout, void *stream) {
    if (!w || !wf) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_flip_weights");
    return omb::unet_flip_weights(w, wf, cin, cout, (cudaStream_t)stream);
}

int omb_unet_avgpool(const void *in, void *out, int32_t X, int32_t Y, int32_t Z, int32_t B, int32_t C,
                     int32_t backward, void *stream) {
    if (!in || !out) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_avgpool");
    return omb::unet_avgpool(in, out, X, Y, Z, B, C, backward, (cudaStream_t)stream);
}

int omb_unet_up_concat(const void *low, const void *skip, void *cat, int32_t X, int32_t Y, int32_t Z, int32_t B,
                       int32_t cl, int32_t cs, void *stream) {
    if (!low || !skip || !cat) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_up_concat");
    return omb::unet_up_concat(low, skip, cat, X, Y, Z, B, cl, cs, (cudaStream_t)stream);
}

int omb_unet_up_concat_bwd(const void *dcat, void *dlow, void *dskip, int32_t X, int32_t Y, int32_t Z, int32_t B,
                           int32_t cl, int32_t cs, void *stream) {
    if (!dcat || !dlow || !dskip) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_up_concat_bwd");
    return omb::unet_up_concat_bwd(dcat, dlow, dskip, X, Y, Z, B, cl, cs, (cudaStream_t)stream);
}

int omb_unet_relu_mask(void *d, const void *a, int64_t n, void *stream) {
    if (!d || !a) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_relu_mask");
    return omb::unet_relu_mask(d, a, n, (cudaStream_t)stream);
}

int omb_unet_make_input(const float *osem, int64_t osem_stride, const float *sens, const float *scale,
                        float sens_scale, void *out, int32_t X, int32_t Y, int32_t Z, int32_t Zs, int32_t B,
                        void *stream) {
    if (!osem || !sens || !scale || !out) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_make_input");
    return omb::unet_make_input(osem, osem_stride, sens, scale, sens_scale, out, X, Y, Z, Zs, B, (cudaStream_t)stream);
}

int omb_unet_head_fwd(const void *a, const void *inp, const float *w, const float *bias, float *pred, int64_t nvox,
                      void *stream) {
    if (!a || !inp || !w || !bias || !pred) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_head_fwd");
    return omb::unet_head_fwd(a, inp, w, bias, pred, nvox, (cudaStream_t)stream);
}

int omb_unet_head_bwd(const void *a, const float *pred, const float *target, int64_t target_stride,
                      const float *tscale, const float *w, void *da, float *dw, float *db, float *loss, int32_t X,
                      int32_t Y, int32_t Z, int32_t Zs, int32_t B, void *stream) {
    if (!a || !pred || !target || !tscale || !w || !da || !dw || !db || !loss)
        return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_head_bwd");
    return omb::unet_head_bwd(a, pred, target, target_stride, tscale, w, da, dw, db, loss, X, Y, Z, Zs, B,
                              (cudaStream_t)stream);
}

int omb_unet_head_out(const float *pred, const float *scale, float *out, int64_t out_stride, float floor_v, int32_t X,
                      int32_t Y, int32_t Z, int32_t Zs, int32_t B, void *stream) {
    if (!pred || !scale || !out) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_head_out");
    return omb::unet_head_out(pred, scale, out, out_stride, floor_v, X, Y, Z, Zs, B, (cudaStream_t)stream);
}

int omb_unet_adam(float *p, float *m, float *v, const float *g, void *p_bf16, int64_t n, float lr, float beta1,
                  float beta2, int32_t step, float eps, void *stream) {
    if (!p || !m || !v || !g) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_adam");
    if (step < 1) return omb::set_error(OMB_ERR_INVALID, "Adam step must be >= 1");
    return omb::unet_adam(p, m, v, g, p_bf16, n, lr, beta1, beta2, step, eps, (cudaStream_t)stream);
}

int omb_unet_to_bf16(const float *a, void *b, int64_t n, void *stream) {
    if (!a || !b) return omb::set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_unet_to_bf16");
    return omb::unet_to_bf16(a, b, n, (cudaStream_t)stream);
}

}  // extern "C"
