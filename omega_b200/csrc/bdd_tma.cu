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
constexpr int kCTACols = 32;  // detector columns of a CTA (kCTACols / C warps of C-column groups)
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
    int2 slices;           // [first, last] slice the CTA's rays can meet
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

template <int NC>
__global__ void k_bdd_fp_tma(const __grid_constant__ CUtensorMap map_img, const __grid_constant__ CUtensorMap map_imgT,
                             Grid g, const float *__restrict__ xy, const float *__restrict__ uv, int nr, int nc,
                             float pitch_y, int64_t proj0, int64_t nproj, const float *__restrict__ img,
                             const float *__restrict__ imgT, float *__restrict__ y) {
    using namespace bt;
    constexpr int kRB = kCTACols / NC;  // warps per CTA
    constexpr float kC = (float)NC;
    __shared__ Shared sh;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int r = blockIdx.x * 32 + threadIdx.x;
    const int cg = blockIdx.y * kRB + threadIdx.y;
    const int64_t p = blockIdx.z;
    const int c0 = cg * NC;
    const bool active = r < nr && c0 < nc && p < nproj;
    const int n_groups = (nc + NC - 1) / NC;

    // corner rays: first/last active row x first/last active column group
    if (tid < 4) {
        const int r_last = min(blockIdx.x * 32 + 31, nr - 1);
        const int g_last = min((int)blockIdx.y * kRB + kRB - 1, n_groups - 1);
        const int rr = (tid & 1) ? r_last : (int)blockIdx.x * 32;
        const int cc = ((tid & 2) ? g_last : (int)blockIdx.y * kRB) * NC;
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
    // the slices any of the CTA's ray groups can meet (the hull over its
    // corner groups); outside them every footprint integral is zero
    if (tid == 0) {
        SliceRange range = slice_range_empty();
        for (int q = 0; q < 4; ++q) {
            const Corner &c = sh.corner[q];
            slice_range_add(range, c.xa0, c.xa1, c.xb0, c.xb1, c.za0, c.za1, c.zb0, c.zb1, nsl, nlat, g.nz, kC);
        }
        sh.slices = slice_range_bounds(range);
    }
    __syncthreads();
    const int j_lo = sh.slices.x, j_hi = sh.slices.y;

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
        for (int s = 0; s < kStages && j_lo + s <= j_hi; ++s) issue(j_lo + s, s);

    BddRay b{};
    float kerroin = 0.f, kerroin8 = 0.f;
    if (active) {
        b = bdd_ray_setup(g, xy, uv, proj0 + p, r, c0, nr, nc, pitch_y);
        kerroin = b.kerroin;
        // the weight belongs to groups of 8 columns (projectorType5.cl:166-174)
        if (NC > 8 && c0 + 8 < nc) kerroin8 = bdd_kerroin(g, xy, uv, proj0 + p, r, c0 + 8, nr, nc, pitch_y, b.ysl);
    }
    const int64_t z_stride = (int64_t)g.nx * g.ny;
    const float *__restrict__ vol = ysl ? img : imgT;
    const float flat = (float)nlat, fz = (float)g.nz;
    const float dlat = ysl ? g.dx : g.dy;
    const int zmax = g.nz - 1;
    float temp[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) temp[c] = 0.f;
    int tries = kWaitTries;

    for (int j = j_lo; j <= j_hi; ++j) {
        const int t = j - j_lo;  // position in the ring's sequence
        const int s = t % kStages;
        if (!mbar_wait(smem_u32(&sh.full[s]), (uint32_t)((t / kStages) & 1), tries)) {
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
        // a run of columns wholly above or below the volume integrates to zero
        if (active && cr > cl && zu < fz && fmaf(kC, w, zu) > 0.f) {
            const float inv_area = 1.f / (fabsf(fmaf(fj, b.dw1, b.dw0)) * dlat * w * g.dz);
            const int i0 = (int)cl;
            const Seg seg = make_seg(cl, cr, i0, min((int)ceilf(cr), nlat) - 1 - i0);
            float bz = fminf(fmaxf(zu, 0.f), fz);
            int kc = min((int)bz, zmax);
            const int k_end = min((int)fminf(fmaxf(fmaf(kC, w, zu), 0.f), fz), zmax);
            const int2 o = sh.origin[s];
            // Fast path: the run lies in the staged box, spans at most 3
            // voxels (no tail loop) and a column is narrower than a voxel row
            // (0.99: margin for rounding), so each column crosses at most one
            // new row -- straight-line code, no loops.
            const bool staged = i0 >= o.x && i0 + seg.n < o.x + kBW && kc >= o.y && k_end < o.y + kBZ;
            if (staged && seg.n <= 2 && w < 0.99f && zu >= 0.f && fmaf(kC, w, zu) < fz) {
                // the same, with the run inside the volume: the clamps of the
                // column edges to [0, nz] and of the row to nz - 1 are identities
                const float *q = sh.box[s] + (kc - o.y) * kBW + (i0 - o.x);
                const float *q1 = q + seg.o1, *q2 = q + seg.o2;
                float R = fmaf(seg.w2, *q2, fmaf(seg.w1, *q1, seg.w0 * q[0]));
                float S = 0.f;
                // the row as an exact float: with bz >= 0 and at most one new
                // row per column, (int)bz > kc is bz >= kc + 1, so no
                // float-to-int conversion per column
                float fkc = (float)kc;
                float Cprev = (bz - fkc) * R;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    bz = fmaf((float)(c + 1), w, zu);
                    if (bz >= fkc + 1.f) {
                        S += R;
                        fkc += 1.f;
                        q += kBW;
                        q1 += kBW;
                        q2 += kBW;
                        R = fmaf(seg.w2, *q2, fmaf(seg.w1, *q1, seg.w0 * q[0]));
                    }
                    const float C = fmaf(bz - fkc, R, S);
                    temp[c] = fmaf(C - Cprev, inv_area, temp[c]);
                    Cprev = C;
                }
            } else if (staged && seg.n <= 2 && w < 0.99f) {
                const float *q = sh.box[s] + (kc - o.y) * kBW + (i0 - o.x);
                float R = fmaf(seg.w2, q[seg.o2], fmaf(seg.w1, q[seg.o1], seg.w0 * q[0]));
                float S = 0.f;
                // min((int)bz, zmax) > kc with bz in [0, nz] is bz >= kc + 1
                // below the last row (the exact-float row as above)
                float fkc = (float)kc;
                const float fzmax = (float)zmax;
                float Cprev = (bz - fkc) * R;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    bz = fminf(fmaxf(fmaf((float)(c + 1), w, zu), 0.f), fz);
                    if (bz >= fkc + 1.f && fkc < fzmax) {
                        S += R;
                        fkc += 1.f;
                        q += kBW;
                        R = fmaf(seg.w2, q[seg.o2], fmaf(seg.w1, q[seg.o1], seg.w0 * q[0]));
                    }
                    const float C = fmaf(bz - fkc, R, S);
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
                for (int c = 0; c < NC; ++c) {
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
        if (threadIdx.x == 0 && threadIdx.y == t % kRB && j + kStages <= j_hi) issue(j + kStages, s);
    }
    if (!active) return;
    const int ncol = min(NC, nc - c0);
    const int64_t idx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
#pragma unroll
    for (int c = 0; c < NC; ++c)
        if (c < ncol) y[idx + (int64_t)c * nr] = temp[c] * (c < 8 ? kerroin : kerroin8);
}

// ---------------------------------------------------------------------------
// Backprojection with the projection data staged by TMA.
//
// Same per-voxel arithmetic as k_bdd_bp<8, ...> (bdd.cu).  A CTA covers 32 x
// 4 voxel columns and a run of kBpZ voxels along z; for projection p its
// voxels' footprints lie in a box of detector rows x columns, found by
// projecting the block's 8 corners (the projective map sends the box to the
// convex hull of their images).  The box of projection p + kStages is loaded
// with cp.async.bulk.tensor while projection p is processed.  Column sums of a
// voxel column whose footprint leaves the box read global memory.
// ---------------------------------------------------------------------------
namespace bb {

constexpr int kThreads = 128;  // 32 x 4 voxel columns
constexpr int kRW = 52;        // detector rows of a box (multiple of 4)
constexpr int kChunk = 16;     // views whose re-based maps the CTA prepares together

// KZ voxels along z per thread (8 or 16)
template <int KZ>
struct Cfg {
    static constexpr int kSlots = bp_slots(KZ);  // prefix-sum slots per thread
    static constexpr int kCW = kSlots + 4;       // detector columns of a box
    static constexpr int kStageFloats = (kRW * kCW + 31) / 32 * 32;  // 128-byte aligned stages
    // the static shared memory stays below 48 KB: 4 stages at 8 voxels, 3 at 16
    static constexpr int kStages = KZ == 8 ? 4 : 3;
    static constexpr int kMinBlocks = KZ == 8 ? 6 : 5;
};

template <int KZ>
struct Shared {
    alignas(128) float box[Cfg<KZ>::kStages][Cfg<KZ>::kStageFloats];
    alignas(8) uint64_t full[Cfg<KZ>::kStages];
    // the maps of a chunk of views re-based to this block, (U0, V0) = the
    // view's box origin; two chunks alternate (the one being consumed and
    // the next, prepared once per kChunk views by all threads)
    BddMapR map[2][kChunk];
    float2 pref[Cfg<KZ>::kSlots][kThreads];
};

}  // namespace bb

template <int KZ, bool SENS, bool FULL>
__global__ void __launch_bounds__(bb::kThreads, bb::Cfg<KZ>::kMinBlocks)
    k_bdd_bp_tma(const __grid_constant__ CUtensorMap map_y, Grid g, const BddProj *__restrict__ pj,
                 const BddMap64 *__restrict__ pm, int nr, int nc, int64_t nproj, const float *__restrict__ y,
                 float *__restrict__ img, float *__restrict__ sens) {
    using namespace bb;
    constexpr int kBpZ = KZ;
    constexpr int kSlots = Cfg<KZ>::kSlots, kCW = Cfg<KZ>::kCW, kStages = Cfg<KZ>::kStages;
    __shared__ Shared<KZ> sh;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int lane = threadIdx.x;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 4 + threadIdx.y;
    const int kz0 = blockIdx.z * kBpZ;
    const bool active = i < g.nx && j < g.ny && kz0 < g.nz;

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bt::smem_u32(&sh.full[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // corner `tid & 7` of the CTA's voxel block (edges of its voxels)
    const int q8 = tid & 7;
    const float cx = g.bx + (float)((q8 & 1) ? min((int)blockIdx.x * 32 + 32, g.nx) : (int)blockIdx.x * 32) * g.dx;
    const float cy = g.by + (float)((q8 & 2) ? min((int)blockIdx.y * 4 + 4, g.ny) : (int)blockIdx.y * 4) * g.dy;
    const float cz = g.bz + (float)((q8 & 4) ? min(kz0 + kBpZ, g.nz) : kz0) * g.dz;
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 4;
    const double p0x = (double)g.bx + (double)i0 * g.dx, p0y = (double)g.by + (double)j0 * g.dy;
    const double p0z = (double)g.bz + (double)kz0 * g.dz;
    // prepares the re-based maps of views [kChunk c, kChunk (c + 1)): thread
    // 8v + q projects corner q of the block with view v's float map, the 8
    // corners' minimum gives the box origin, and thread 8v re-bases the FP64
    // map to it.  All threads of the CTA take part (warp-uniform shuffles).
    auto prepare = [&](int64_t c) {
        const int64_t pv = c * kChunk + (tid >> 3);
        const bool have = pv < nproj;
        const BddProj P = pj[have ? pv : 0];
        float2 uv = bdd_corner_uv(P, cx, cy, cz);
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            uv.x = fminf(uv.x, __shfl_xor_sync(0xffffffffu, uv.x, o));
            uv.y = fminf(uv.y, __shfl_xor_sync(0xffffffffu, uv.y, o));
        }
        if (have && q8 == 0) {
            const int2 org = bdd_block_origin(uv.x, uv.y, nr, nc);
            bdd_rebase(sh.map[c & 1][tid >> 3], pm[pv], P, p0x, p0y, p0z, org.x, org.y);
        }
    };
    // loads the detector box of projection pn into stage s (one thread)
    auto produce = [&](int64_t pn, int s) {
        const BddMapR &M = sh.map[(pn / kChunk) & 1][pn % kChunk];
        const uint32_t bar = bt::smem_u32(&sh.full[s]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                     "r"((uint32_t)(kRW * kCW * sizeof(float)))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
            "%4}], [%5];\n" ::"r"(bt::smem_u32(sh.box[s])),
            "l"(reinterpret_cast<uint64_t>(&map_y)), "r"(M.o.x), "r"(M.o.y), "r"((int)pn), "r"(bar)
            : "memory");
    };
    prepare(0);
    __syncthreads();
    if (tid == 0)
        for (int s = 0; s < kStages && s < nproj; ++s) produce(s, s);

    const int nzt = FULL ? kBpZ : min(kBpZ, g.nz - kz0);
    // voxel centre relative to the block corner (exact for grid steps)
    const float rx0 = ((float)(i - i0) + 0.5f) * g.dx;
    const float ry0 = ((float)(j - j0) + 0.5f) * g.dy;
    const float rz0 = 0.5f * g.dz;
    const float qx = fmaf((float)i, g.dx, g.bx + 0.5f * g.dx);
    const float qy = fmaf((float)j, g.dy, g.by + 0.5f * g.dy);
    const float qz0 = fmaf((float)kz0, g.dz, g.bz + 0.5f * g.dz);
    const float hx = 0.5f * g.dx, hy = 0.5f * g.dy, hz = 0.5f * g.dz;
    const float fnc = (float)nc;
    float temp[kBpZ], wsum[kBpZ];
#pragma unroll
    for (int t = 0; t < kBpZ; ++t) {
        temp[t] = 0.f;
        wsum[t] = 0.f;
    }
    int tries = bt::kWaitTries;
    for (int64_t p = 0; p < nproj; ++p) {
        const int s = (int)(p % kStages);
        // the next chunk's maps, kChunk views ahead of their first use (the
        // buffer held the previous chunk, all of whose views are done)
        if (p % kChunk == 0 && p + kChunk < nproj) prepare(p / kChunk + 1);
        if (!bt::mbar_wait(bt::smem_u32(&sh.full[s]), (uint32_t)((p / kStages) & 1), tries)) {
            atomicExch(&g_device_error, 1);
            tries = bt::kWaitTriesAfterFailure;
        }
        do {
            if (!active) break;
            // u, v below are relative to the box origin (U0, V0)
            const BddMapR M = sh.map[(p / kChunk) & 1][p % kChunk];
            BpFootprint F;
            if (!bdd_bp_footprint(M, rx0, ry0, rz0, hx, hy, hz, qx, qy, g, nr, nc, nzt, F)) break;
            const Seg &seg = F.seg;
            const int r0 = F.r0, cA = F.cA, ncols = F.ncols;
            const float V0 = F.V0, vl0 = F.vl0, vr0 = F.vr0, svl = F.svl, svr = F.svr;
            const float axy = F.axy, kscale = F.kscale;
            const bool staged = r0 >= 0 && r0 + seg.n < kRW && cA >= 0 && cA + ncols <= kCW;
            if (ncols <= kSlots) {
                float acc = 0.f;
                float2 *pw = &sh.pref[0][tid];
                if (staged && seg.n <= 2) {
                    const float *q0 = sh.box[s] + cA * kRW + r0;
                    const float *q1 = q0 + seg.o1, *q2 = q0 + seg.o2;
#pragma unroll
                    for (int m = 0; m < kSlots; ++m) {
                        if (m >= ncols) break;
                        const float rs = fmaf(seg.w2, q2[m * kRW], fmaf(seg.w1, q1[m * kRW], seg.w0 * q0[m * kRW]));
                        pw[m * kThreads] = bp_prefix_node(acc, rs, m);
                        acc += rs;
                    }
                } else {
                    const float *yp = y + p * (int64_t)nr * nc + (int64_t)M.o.y * nr + M.o.x + r0;
#pragma unroll
                    for (int m = 0; m < kSlots; ++m) {
                        if (m >= ncols) break;
                        const float rs = seg_sum(seg, yp + (int64_t)(cA + m) * nr);
                        pw[m * kThreads] = bp_prefix_node(acc, rs, m);
                        acc += rs;
                    }
                }
                bp_voxels<kBpZ, SENS, FULL, kThreads>(F, &sh.pref[0][tid], nzt, nc, qz0 - M.s.z, g.dz, temp, wsum);
            } else {
                const float *yp = y + p * (int64_t)nr * nc + (int64_t)M.o.y * nr + M.o.x + r0;
#pragma unroll
                for (int t = 0; t < kBpZ; ++t) {
                    const float vlt = fmaf((float)t, svl, vl0), vrt = fmaf((float)t, svr, vr0);
                    const float va = fmaxf(fminf(vlt, vrt), -V0), vb = fminf(fmaxf(vlt, vrt), fnc - V0);
                    if ((FULL || t < nzt) && vb > va) {
                        const int c0 = (int)floorf(va), c1 = min((int)ceilf(vb), nc - M.o.y) - 1;
                        float apu = 0.f;
                        for (int c = c0; c <= c1; ++c) {
                            const float ov = fminf(vb, (float)(c + 1)) - fmaxf(va, (float)c);
                            apu = fmaf(ov, seg_sum(seg, yp + (int64_t)c * nr), apu);
                        }
                        if (apu != 0.f) {
                            const float vz = fmaf((float)t, g.dz, qz0) - M.s.z;
                            const float q2 = fmaf(vz, vz, axy);
                            const float ker = kscale * (q2 * rsqrtf(q2));
                            temp[t] = fmaf(apu, ker, temp[t]);
                            if (SENS) wsum[t] += ker;
                        }
                    }
                }
            }
        } while (false);
        __syncthreads();  // stage s is free again
        if (lane == 0 && threadIdx.y == (int)(p % 4) && p + kStages < nproj) produce(p + kStages, s);
    }
    if (!active) return;
    int64_t n = i + (int64_t)j * g.nx + (int64_t)kz0 * g.nx * g.ny;
#pragma unroll
    for (int t = 0; t < kBpZ; ++t) {
        if (t < nzt) {
            img[n] = temp[t];
            if (SENS) sens[n] = wsum[t];
        }
        n += (int64_t)g.nx * g.ny;
    }
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
                    int64_t nproj, const float *img, const float *imgT, float *y, int cols, cudaStream_t st) {
    CUtensorMap m_img, m_imgT;
    if (!encode_volume(m_img, img, g.nx, g.ny, g.nz) || !encode_volume(m_imgT, imgT, g.ny, g.nx, g.nz))
        return set_error(OMB_ERR_CUDA, "cuTensorMapEncodeTiled failed for the type-5 image maps");
    const int C = cols == 16 ? 16 : 8;
    const int rb = bt::kCTACols / C;
    const int groups = (nc + C - 1) / C;
    dim3 block(32, rb);
    dim3 grid((nr + 31) / 32, (groups + rb - 1) / rb, (unsigned)nproj);
    if (C == 16)
        k_bdd_fp_tma<16><<<grid, block, 0, st>>>(m_img, m_imgT, g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y);
    else
        k_bdd_fp_tma<8><<<grid, block, 0, st>>>(m_img, m_imgT, g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y);
    OMB_LAUNCH_CHECK("type-5 TMA forward launch");
    return OMB_OK;
}

bool bdd_bp_tma_supported(int nr, const float *y) {
    return nr % 4 == 0 && ((uintptr_t)y & 15) == 0 && encode_fn() != nullptr;
}

template <int KZ>
static int launch_bp_tma(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj,
                         const float *y, float *img, float *sens, cudaStream_t st) {
    auto fn = encode_fn();
    CUtensorMap m_y;
    const cuuint64_t dims[3] = {(cuuint64_t)nr, (cuuint64_t)nc, (cuuint64_t)nproj};
    const cuuint64_t strides[2] = {(cuuint64_t)nr * sizeof(float), (cuuint64_t)nr * nc * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)bb::kRW, (cuuint32_t)bb::Cfg<KZ>::kCW, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    if (!fn || fn(&m_y, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(y), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return set_error(OMB_ERR_CUDA, "cuTensorMapEncodeTiled failed for the type-5 projection map");
    dim3 block(32, 4);
    dim3 grid((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + KZ - 1) / KZ);
    const bool full = g.nz % KZ == 0;
    if (sens && full)
        k_bdd_bp_tma<KZ, true, true><<<grid, block, 0, st>>>(m_y, g, pj, pm, nr, nc, nproj, y, img, sens);
    else if (sens)
        k_bdd_bp_tma<KZ, true, false><<<grid, block, 0, st>>>(m_y, g, pj, pm, nr, nc, nproj, y, img, sens);
    else if (full)
        k_bdd_bp_tma<KZ, false, true><<<grid, block, 0, st>>>(m_y, g, pj, pm, nr, nc, nproj, y, img, sens);
    else
        k_bdd_bp_tma<KZ, false, false><<<grid, block, 0, st>>>(m_y, g, pj, pm, nr, nc, nproj, y, img, sens);
    OMB_LAUNCH_CHECK("type-5 TMA backward launch");
    return OMB_OK;
}

int bdd_backward_tma(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj,
                     const float *y, float *img, float *sens, int kz, cudaStream_t st) {
    if (nproj <= 0) return OMB_OK;
    if (kz == 16) return launch_bp_tma<16>(g, pj, pm, nr, nc, nproj, y, img, sens, st);
    if (kz == 8) return launch_bp_tma<8>(g, pj, pm, nr, nc, nproj, y, img, sens, st);
    return set_error(OMB_ERR_INVALID, "the staged type-5 backprojection takes runs of 8 or 16 voxels");
}

int take_device_error() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)) != cudaSuccess) return -1;
    const int zero = 0;
    if (v != 0 && cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)) != cudaSuccess) return -1;
    return v;
}

}  // namespace omb
