// Type-5 (branchless distance-driven) forward projection with the image
// patches staged by the tensor memory accelerator.
//
// Same per-ray arithmetic as k_bdd_fp<8> (bdd.cu): thread = (detector row,
// group of 8 columns, projection), slices along the dominant source axis, one
// row integral per voxel row the 8 column footprints cross.  What changes is
// where the voxels come from.  A CTA covers 32 detector rows x kRB groups of 8
// columns of one projection; on slice j its rays' footprints lie inside a
// small box of the slice (lateral x z), found from the CTA's four corner rays
// (the footprint edges are monotonic along the panel).  One thread per slice
// loads that box with cp.async.bulk.tensor into a kStages-deep ring of
// shared-memory buffers, kStages - 1 slices ahead of the compute, completing
// on an mbarrier; the row integrals then read shared memory.  A ray whose
// footprint leaves the box on some slice (geometries the box was not sized
// for) reads that slice from global memory instead, with the same arithmetic,
// so results do not depend on the staging.
//
// Every mbarrier wait is bounded; a wait that runs out sets the device error
// word read by omb_take_device_error() and later waits give up quickly, so
// the kernel always ends.  Tensor-map loads only (no stores, no multicast); the
// box's lateral start is a multiple of 4 floats (16 bytes).
#include <cuda.h>
#include <cudaTypedefs.h>

#include "bdd.cuh"
#include "kernels.h"

namespace omb {

__device__ int g_device_error = 0;

namespace bt {

constexpr int kBW = 40;       // lateral voxels of a staged box (x multiple of 4: 16-byte aligned starts)
constexpr int kBZ = 36;       // voxel rows (z) of a staged box
constexpr int kStages = 4;    // ring depth
constexpr int kRB = 4;        // warps per CTA = groups of 8 columns
constexpr int kBoxFloats = kBW * kBZ;
constexpr int kWaitTries = 1 << 22;
constexpr int kWaitTriesAfterFailure = 64;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int tries) {
    for (int i = 0; i < tries; ++i) {
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

// Footprint lines of one corner ray (the BddRay fields the box needs).
struct Corner {
    float xa0, xa1, xb0, xb1, za0, za1, zb0, zb1, dz0, dz1;
};

struct Shared {
    alignas(128) float box[kStages][kBoxFloats];
    alignas(8) uint64_t full[kStages];
    int2 origin[kStages];  // (lateral, z) voxel of the box's first element
    Corner corner[4];
};

// Box of slice j covering the four corner rays' footprints (lateral start
// rounded down to a multiple of 4), clamped into the volume.
__device__ __forceinline__ int2 slice_box(const Shared &sh, int j, int nlat, int nz) {
    const float fj = (float)j;
    float lo = 3.4e38f, zlo = 3.4e38f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const Corner &c = sh.corner[q];
        const float xa = fmaf(fj, c.xa1, c.xa0), xb = fmaf(fj, c.xb1, c.xb0);
        const float za = fmaf(fj, c.za1, c.za0), zb = fmaf(fj, c.zb1, c.zb0);
        lo = fminf(lo, fminf(xa, xb));
        zlo = fminf(zlo, fminf(za, zb));
    }
    int x = (int)floorf(fmaxf(lo - 0.5f, 0.f));
    x = min(x, max(nlat - 1, 0)) & ~3;
    int z = (int)floorf(fmaxf(zlo - 0.5f, 0.f));
    z = min(z, nz - 1);
    return make_int2(x, z);
}

}  // namespace bt

__global__ void k_bdd_fp_tma(const __grid_constant__ CUtensorMap map_img, const __grid_constant__ CUtensorMap map_imgT,
                             Grid g, const float *__restrict__ xy, const float *__restrict__ uv, int nr, int nc,
                             float pitch_y, int64_t proj0, int64_t nproj, const float *__restrict__ img,
                             const float *__restrict__ imgT, float *__restrict__ y) {
    using namespace bt;
    __shared__ Shared sh;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int r = blockIdx.x * 32 + threadIdx.x;
    const int cg = blockIdx.y * kRB + threadIdx.y;
    const int64_t p = blockIdx.z;
    const int c0 = cg * 8;
    const bool active = r < nr && c0 < nc && p < nproj;
    const int n_groups = (nc + 7) / 8;

    // corner rays: first/last active row x first/last active column group
    if (tid < 4) {
        const int r_last = min(blockIdx.x * 32 + 31, nr - 1);
        const int g_last = min((int)blockIdx.y * kRB + kRB - 1, n_groups - 1);
        const int rr = (tid & 1) ? r_last : (int)blockIdx.x * 32;
        const int cc = ((tid & 2) ? g_last : (int)blockIdx.y * kRB) * 8;
        const BddRay b = bdd_ray_setup(g, xy, uv, proj0 + p, rr, cc, nr, nc, pitch_y);
        sh.corner[tid] = Corner{b.xa0, b.xa1, b.xb0, b.xb1, b.za0, b.za1, b.zb0, b.zb1, b.dz0, b.dz1};
        if (tid == 0) {
            for (int s = 0; s < kStages; ++s)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&sh.full[s])) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
    }
    __syncthreads();

    // slice orientation is uniform over the CTA (one projection)
    const float *q6 = xy + (proj0 + p) * 6;
    const bool ysl = fabsf(__ldg(q6)) <= fabsf(__ldg(q6 + 1));
    const int nsl = ysl ? g.ny : g.nx;
    const int nlat = ysl ? g.nx : g.ny;
    const CUtensorMap *map = ysl ? &map_img : &map_imgT;

    // loads slice jn into stage s (one thread)
    auto issue = [&](int jn, int s) {
        const int2 o = slice_box(sh, jn, nlat, g.nz);
        sh.origin[s] = o;
        const uint32_t bar = smem_u32(&sh.full[s]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                     "r"((uint32_t)(kBoxFloats * sizeof(float)))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
            "[%5];\n" ::"r"(smem_u32(sh.box[s])),
            "l"(reinterpret_cast<uint64_t>(map)), "r"(o.x), "r"(jn), "r"(o.y), "r"(bar)
            : "memory");
    };
    if (tid == 0)
        for (int s = 0; s < kStages && s < nsl; ++s) issue(s, s);

    BddRay b{};
    float kerroin = 0.f;
    if (active) {
        b = bdd_ray_setup(g, xy, uv, proj0 + p, r, c0, nr, nc, pitch_y);
        kerroin = b.kerroin;
    }
    const int64_t z_stride = (int64_t)g.nx * g.ny;
    const float *__restrict__ vol = ysl ? img : imgT;
    const float flat = (float)nlat, fz = (float)g.nz;
    const float dlat = ysl ? g.dx : g.dy;
    const int zmax = g.nz - 1;
    float temp[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) temp[c] = 0.f;
    int tries = kWaitTries;

    for (int j = 0; j < nsl; ++j) {
        const int s = j % kStages;
        if (!mbar_wait(smem_u32(&sh.full[s]), (uint32_t)((j / kStages) & 1), tries)) {
            atomicExch(&g_device_error, 1);
            tries = kWaitTriesAfterFailure;
        }
        const float fj = (float)j;
        const float xa = fmaf(fj, b.xa1, b.xa0), xb = fmaf(fj, b.xb1, b.xb0);
        const float za = fmaf(fj, b.za1, b.za0), zb = fmaf(fj, b.zb1, b.zb0);
        const float el = fminf(xa, xb), er = fmaxf(xa, xb);
        const float zu = fminf(za, zb);
        const float w = fabsf(fmaf(fj, b.dz1, b.dz0));
        const float cl = fmaxf(el, 0.f), cr = fminf(er, flat);
        if (active && cr > cl) {
            const float inv_area = 1.f / (fabsf(fmaf(fj, b.dw1, b.dw0)) * dlat * w * g.dz);
            const int i0 = (int)cl;
            const Seg seg = make_seg(cl, cr, i0, min((int)ceilf(cr), nlat) - 1 - i0);
            float bz = fminf(fmaxf(zu, 0.f), fz);
            int kc = min((int)bz, zmax);
            const int k_end = min((int)fminf(fmaxf(fmaf(8.f, w, zu), 0.f), fz), zmax);
            const int2 o = sh.origin[s];
            // Fast path: the run lies in the staged box, spans at most 3
            // voxels (no tail loop) and a column is narrower than a voxel row
            // (0.99: margin for rounding), so each column crosses at most one
            // new row -- straight-line code, no loops.
            const bool staged = i0 >= o.x && i0 + seg.n < o.x + kBW && kc >= o.y && k_end < o.y + kBZ;
            if (staged && seg.n <= 2 && w < 0.99f) {
                const float *q = sh.box[s] + (kc - o.y) * kBW + (i0 - o.x);
                float R = fmaf(seg.w2, q[seg.o2], fmaf(seg.w1, q[seg.o1], seg.w0 * q[0]));
                float S = 0.f;
                float Cprev = (bz - (float)kc) * R;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    bz = fminf(fmaxf(fmaf((float)(c + 1), w, zu), 0.f), fz);
                    const int kn = min((int)bz, zmax);
                    if (kc < kn) {
                        S += R;
                        ++kc;
                        q += kBW;
                        R = fmaf(seg.w2, q[seg.o2], fmaf(seg.w1, q[seg.o1], seg.w0 * q[0]));
                    }
                    const float C = fmaf(bz - (float)kc, R, S);
                    temp[c] = fmaf(C - Cprev, inv_area, temp[c]);
                    Cprev = C;
                }
            } else {
                const float *box = sh.box[s] + (i0 - o.x) - o.y * kBW;
                const float *slice = vol + (int64_t)j * nlat + i0;
#define row_integral(k) \
    (staged ? seg_sum_shared(seg, box + (k) * kBW) : seg_sum(seg, slice + (int64_t)(k) * z_stride))
                float R = row_integral(kc);
                float S = 0.f;
                float Cprev = (bz - (float)kc) * R;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    bz = fminf(fmaxf(fmaf((float)(c + 1), w, zu), 0.f), fz);
                    const int kn = min((int)bz, zmax);
                    while (kc < kn) {
                        S += R;
                        R = row_integral(++kc);
                    }
                    const float C = fmaf(bz - (float)kc, R, S);
                    temp[c] = fmaf(C - Cprev, inv_area, temp[c]);
                    Cprev = C;
                }
#undef row_integral
            }
        }
        __syncthreads();  // stage s is free again
        if (threadIdx.x == 0 && threadIdx.y == j % kRB && j + kStages < nsl) issue(j + kStages, s);
    }
    if (!active) return;
    const int ncol = min(8, nc - c0);
    const int64_t idx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
#pragma unroll
    for (int c = 0; c < 8; ++c)
        if (c < ncol) y[idx + (int64_t)c * nr] = temp[c] * kerroin;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

// 3-D map of a volume stored (lat, slice, z) with lat fastest; box kBW x 1 x kBZ.
static bool encode_volume(CUtensorMap &m, const float *base, int nlat, int nsl, int nz) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nlat, (cuuint64_t)nsl, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nlat * sizeof(float), (cuuint64_t)nlat * nsl * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)bt::kBW, 1u, (cuuint32_t)bt::kBZ};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    return fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool bdd_fp_tma_supported(const Grid &g, const float *img, const float *imgT) {
    // row strides must be multiples of 16 bytes and the bases 16-byte aligned
    return g.nx % 4 == 0 && g.ny % 4 == 0 && ((uintptr_t)img & 15) == 0 && ((uintptr_t)imgT & 15) == 0 &&
           encode_fn() != nullptr;
}

int bdd_forward_tma(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                    int64_t nproj, const float *img, const float *imgT, float *y, cudaStream_t st) {
    CUtensorMap m_img, m_imgT;
    if (!encode_volume(m_img, img, g.nx, g.ny, g.nz) || !encode_volume(m_imgT, imgT, g.ny, g.nx, g.nz))
        return set_error(OMB_ERR_CUDA, "cuTensorMapEncodeTiled failed for the type-5 image maps");
    const int groups = (nc + 7) / 8;
    dim3 block(32, bt::kRB);
    dim3 grid((nr + 31) / 32, (groups + bt::kRB - 1) / bt::kRB, (unsigned)nproj);
    k_bdd_fp_tma<<<grid, block, 0, st>>>(m_img, m_imgT, g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y);
    OMB_LAUNCH_CHECK("type-5 TMA forward launch");
    return OMB_OK;
}

int take_device_error() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)) != cudaSuccess) return -1;
    const int zero = 0;
    if (v != 0 && cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)) != cudaSuccess) return -1;
    return v;
}

}  // namespace omb
