// Projector type 5: branchless distance-driven (BDD) forward and
// backprojection for flat-panel cone-beam CT.
//
// The reference (projectorType5.cl:64-333 forward, 381-757 backward)
// integrates the image over each detector pixel's footprint on every slice,
// and the measurement over each voxel's footprint on the detector, by
// sampling summed-area tables through linear-filtered textures.  Those SAT
// differences are the exact footprint integrals of the piecewise-constant
// image; here the same integrals are formed directly from the voxels /
// pixels the footprint overlaps, with exact overlap lengths:
//  * no summed-area tables are built per call;
//  * FP32 stays accurate (SAT differences of large cumulative sums cancel,
//    and texture filtering weights have 8 fractional bits);
//  * the image (<= 80 MB here) is read from L2 instead of two SAT volumes.
// Footprint geometry follows the reference exactly: detector-pixel corner
// rays dL/dR/dU/dD (getDetectorCoordinatesCT, general_opencl_functions.h:
// 1363-1406), slices along the dominant source axis, 8 detector columns per
// thread stepping the footprint by its own width; voxel mid-plane corners
// LU/RD projected to the panel plane in the backprojection, weights
// dx*dy*dz/|u| (forward) and d*|v|/|v_axis| (backward), backprojection
// sensitivity summed only where the footprint integral is nonzero.
#include "bdd.cuh"
#include "kernels.h"

namespace omb {


// Forward projection.  Thread = (detector row, group of 8 columns, projection).
// `img` is x-fastest, `imgT` the same image y-fastest; slices along y read
// `img`, slices along x read `imgT`, so a warp's 32 rows read consecutive
// addresses in both cases.
template <int kColsPerThread>
__global__ void k_bdd_fp(Grid g, const float *__restrict__ xy, const float *__restrict__ uv,
                                                int nr, int nc, float pitch_y, int64_t proj0, int64_t nproj,
                                                const float *__restrict__ img, const float *__restrict__ imgT,
                                                float *__restrict__ y) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int cg = blockIdx.y * blockDim.y + threadIdx.y;
    const int64_t p = blockIdx.z;
    const int c0 = cg * kColsPerThread;
    if (r >= nr || c0 >= nc || p >= nproj) return;
    const int ncol = min(kColsPerThread, nc - c0);
    const BddRay b = bdd_ray_setup(g, xy, uv, proj0 + p, r, c0, nr, nc, pitch_y);
    // The weight belongs to groups of 8 columns, taken at each group's first
    // column (projectorType5.cl:166-174, 327-331): a 16-column thread holds two.
    const float kerroin8 =
        kColsPerThread > 8 && c0 + 8 < nc ? bdd_kerroin(g, xy, uv, proj0 + p, r, c0 + 8, nr, nc, pitch_y, b.ysl) : 0.f;
    const int nsl = b.ysl ? g.ny : g.nx;       // slices
    const int nlat = b.ysl ? g.nx : g.ny;      // voxels across a slice
    const int64_t sl_stride = nlat;
    const int64_t z_stride = (int64_t)g.nx * g.ny;
    const float *__restrict__ vol = b.ysl ? img : imgT;
    const float flat = (float)nlat, fz = (float)g.nz;
    const float dlat = b.ysl ? g.dx : g.dy;
    float temp[kColsPerThread];
#pragma unroll
    for (int c = 0; c < kColsPerThread; ++c) temp[c] = 0.f;

    const int zmax = g.nz - 1;
    // only the slices where the group's footprint can meet the volume
    SliceRange range = slice_range_empty();
    slice_range_add(range, b.xa0, b.xa1, b.xb0, b.xb1, b.za0, b.za1, b.zb0, b.zb1, nsl, nlat, g.nz,
                    (float)kColsPerThread);
    const int2 jr = slice_range_bounds(range);
    for (int j = jr.x; j <= jr.y; ++j) {
        const float fj = (float)j;
        const float xa = fmaf(fj, b.xa1, b.xa0), xb = fmaf(fj, b.xb1, b.xb0);
        const float za = fmaf(fj, b.za1, b.za0), zb = fmaf(fj, b.zb1, b.zb0);
        const float el = fminf(xa, xb), er = fmaxf(xa, xb);
        const float zu = fminf(za, zb);
        const float w = fabsf(fmaf(fj, b.dz1, b.dz0));
        // lateral overlap range (clamped to the slice); a run of columns wholly
        // above or below the volume integrates to exactly zero
        const float cl = fmaxf(el, 0.f), cr = fminf(er, flat);
        if (!(cr > cl) || !(zu < fz) || !(fmaf((float)kColsPerThread, w, zu) > 0.f)) continue;
        const float inv_area = 1.f / (fabsf(fmaf(fj, b.dw1, b.dw0)) * dlat * w * g.dz);
        const int i0 = (int)cl;  // cl >= 0: truncation is floor
        const Seg seg = make_seg(cl, cr, i0, min((int)ceilf(cr), nlat) - 1 - i0);
        const float *slice = vol + (int64_t)j * sl_stride + i0;
#define row_integral(k) seg_sum(seg, slice + (int64_t)(k) * z_stride)
        // The 8 columns partition [zu, zu + 8w] along z.  With C(b) the
        // integral of the lateral row integrals from zu up to b, column c is
        // C(b_{c+1}) - C(b_c): walk b_0 < ... < b_8 and the voxel rows
        // together, one row integral per row crossed.
        float bz = fminf(fmaxf(zu, 0.f), fz);
        int kc = min((int)bz, zmax);
        float R = row_integral(kc);
        float S = 0.f;
        float Cprev = (bz - (float)kc) * R;
#pragma unroll
        for (int c = 0; c < kColsPerThread; ++c) {
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
    }
#undef row_integral
    int64_t idx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
#pragma unroll
    for (int c = 0; c < kColsPerThread; ++c)
        if (c < ncol) y[idx + (int64_t)c * nr] = temp[c] * (c < 8 ? b.kerroin : kerroin8);
}

// Ray-driven (scatter) backprojection: the exact adjoint of k_bdd_fp<8>.
// Same thread layout and footprint walk as the forward projection; where the
// forward sums the lateral row integrals of the rows a column's axial range
// [b_c, b_c+1] crosses, weighted by the overlap lengths, the adjoint collects
// for every crossed row k the measurement-weighted overlaps
//   A(k) = kerroin * sum_c y_c * |[b_c, b_c+1] n [k, k+1]|
// and adds A(k) * w_i / area to the voxels i of the lateral run.  Float
// atomics, or (FIXED) int64 atomics of round-toward-zero(v * 1e11): the sum
// of integers does not depend on the order the atomics land in, so the
// fixed-point image is bit-identical run to run.  SENS adds A^T 1.
template <bool FIXED, bool SENS>
__global__ void k_bdd_bp_ray(Grid g, const float *__restrict__ xy, const float *__restrict__ uv, int nr, int nc,
                             float pitch_y, int64_t proj0, int64_t nproj, const float *__restrict__ y,
                             float *__restrict__ img, float *__restrict__ sens, unsigned long long *__restrict__ acc,
                             unsigned long long *__restrict__ acc_s) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int cg = blockIdx.y * blockDim.y + threadIdx.y;
    const int64_t p = blockIdx.z;
    const int c0 = cg * 8;
    if (r >= nr || c0 >= nc || p >= nproj) return;
    const int ncol = min(8, nc - c0);
    const int64_t idx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
    float yv[8];
    bool any = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        yv[c] = c < ncol ? __ldg(y + idx + (int64_t)c * nr) : 0.f;
        any |= yv[c] != 0.f;
    }
    if (!SENS && !any) return;
    const BddRay b = bdd_ray_setup(g, xy, uv, proj0 + p, r, c0, nr, nc, pitch_y);
    const int nsl = b.ysl ? g.ny : g.nx;
    const int nlat = b.ysl ? g.nx : g.ny;
    // slices along y: lateral = x; slices along x: lateral = y (x-fastest image)
    const int64_t lat_stride = b.ysl ? 1 : g.nx;
    const int64_t sl_stride = b.ysl ? g.nx : 1;
    const int64_t z_stride = (int64_t)g.nx * g.ny;
    const float flat = (float)nlat, fz = (float)g.nz;
    const float dlat = b.ysl ? g.dx : g.dy;
    const int zmax = g.nz - 1;
    const float ker = b.kerroin;
    SliceRange range = slice_range_empty();
    slice_range_add(range, b.xa0, b.xa1, b.xb0, b.xb1, b.za0, b.za1, b.zb0, b.zb1, nsl, nlat, g.nz, 8.f);
    const int2 jr = slice_range_bounds(range);

    for (int j = jr.x; j <= jr.y; ++j) {
        const float fj = (float)j;
        const float xa = fmaf(fj, b.xa1, b.xa0), xb = fmaf(fj, b.xb1, b.xb0);
        const float za = fmaf(fj, b.za1, b.za0), zb = fmaf(fj, b.zb1, b.zb0);
        const float el = fminf(xa, xb), er = fmaxf(xa, xb);
        const float zu = fminf(za, zb);
        const float w = fabsf(fmaf(fj, b.dz1, b.dz0));
        const float cl = fmaxf(el, 0.f), cr = fminf(er, flat);
        if (!(cr > cl) || !(zu < fz) || !(fmaf(8.f, w, zu) > 0.f)) continue;
        const float inv_area = 1.f / (fabsf(fmaf(fj, b.dw1, b.dw0)) * dlat * w * g.dz);
        const int i0 = (int)cl;
        const Seg seg = make_seg(cl, cr, i0, min((int)ceilf(cr), nlat) - 1 - i0);
        const int64_t base = (int64_t)j * sl_stride + (int64_t)i0 * lat_stride;
        const float scale = ker * inv_area;
        // the row's accumulated weight goes to the lateral run's voxels
        auto flush = [&](int k, float A, float As) {
            const int64_t row = base + (int64_t)k * z_stride;
            for (int e = 0; e <= seg.n; ++e) {
                const float we = e == 0 ? seg.w0 : (e == 1 ? seg.w1 : (e == 2 ? seg.w2 :
                                 fminf(seg.hi, (float)(seg.base + e + 1)) - (float)(seg.base + e)));
                const int64_t off = row + (int64_t)e * lat_stride;
                const float v = A * scale * we;
                if (FIXED) {
                    if (v != 0.f) atomicAdd(acc + off, (unsigned long long)(long long)((double)v * kFixedScale));
                    if (SENS) {
                        const float vs = As * scale * we;
                        if (vs != 0.f) atomicAdd(acc_s + off, (unsigned long long)(long long)((double)vs * kFixedScale));
                    }
                } else {
                    if (v != 0.f) atomicAdd(img + off, v);
                    if (SENS) {
                        const float vs = As * scale * we;
                        if (vs != 0.f) atomicAdd(sens + off, vs);
                    }
                }
            }
        };
        float bz = fminf(fmaxf(zu, 0.f), fz);
        int kc = min((int)bz, zmax);
        float prev = bz, A = 0.f, As = 0.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float bzn = fminf(fmaxf(fmaf((float)(c + 1), w, zu), 0.f), fz);
            const int kn = min((int)bzn, zmax);
            const float one = c < ncol ? 1.f : 0.f;
            while (kc < kn) {
                const float len = (float)(kc + 1) - prev;
                A = fmaf(yv[c], len, A);
                if (SENS) As = fmaf(one, len, As);
                flush(kc, A, As);
                A = 0.f;
                As = 0.f;
                ++kc;
                prev = (float)kc;
            }
            const float len = bzn - prev;
            A = fmaf(yv[c], len, A);
            if (SENS) As = fmaf(one, len, As);
            prev = bzn;
        }
        flush(kc, A, As);
    }
}

// y-fastest copy of an x-fastest volume (per z slice, a 2-D transpose).
__global__ void k_transpose_xy(const float *__restrict__ in, float *__restrict__ out, int nx, int ny, int nz) {
    __shared__ float tile[32][33];
    const int z = blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const int64_t zo = (int64_t)z * nx * ny;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const int x = x0 + threadIdx.x, y = y0 + yy;
        if (x < nx && y < ny) tile[yy][threadIdx.x] = in[zo + x + (int64_t)y * nx];
    }
    __syncthreads();
    for (int xx = threadIdx.y; xx < 32; xx += blockDim.y) {
        const int y = y0 + threadIdx.x, x = x0 + xx;
        if (x < nx && y < ny) out[zo + y + (int64_t)x * ny] = tile[threadIdx.x][xx];
    }
}

// ---------------------------------------------------------------------------
// Backprojection.
// Per projection, a projective map from world coordinates to continuous
// detector pixel-edge coordinates (u along rows, v along columns):
//   u = (au . q + au0) / (c . q + c0),  v = (av . q + av0) / (c . q + c0)
// normalised so the denominator is 1 at the world origin.  Built on the host
// in FP64 from the same source, panel and direction vectors the reference's
// computeGeom5 uses (omegatomo/projector/init.py:6-37).
// ---------------------------------------------------------------------------


// Voxel-driven backprojection, kBpZ voxels along z per thread.  For the flat
// panels of this path (rows in the xy-plane, columns along z) the detector
// row coordinate u and the projective denominator do not depend on z, so the
// row footprint [ua, ub] and its weights are formed once per projection and
// shared by the thread's voxels.  The row-weighted column sums RS_c over the
// columns the voxel run covers are accumulated into prefix sums P_c (kept in
// shared memory, one slot column per thread); the footprint integral of a
// voxel over [va, vb] is then D(vb) - D(va) with D(v) = P_m + (v - m) RS_m,
// m = floor(v): two shared-memory reads per voxel instead of a walk over its
// detector pixels.
template <int kBpZ, bool SENS, bool FULL, int kBpThreads>
__global__ void k_bdd_bp(Grid g, const BddProj *__restrict__ pj, const BddMap64 *__restrict__ pm, int nr, int nc,
                         int64_t nproj, const float *__restrict__ y, float *__restrict__ img,
                         float *__restrict__ sens) {
    constexpr int kBpCols = bp_slots(kBpZ);
    __shared__ float2 pref[kBpCols][kBpThreads];  // (P_m, RS_m) of column cA + m
    __shared__ BddMapR smap[2];                   // the projection's map re-based to this block (double-buffered)
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int i0 = blockIdx.x * blockDim.x, j0 = blockIdx.y * blockDim.y;
    const int i = i0 + threadIdx.x;
    const int j = j0 + threadIdx.y;
    const int kz0 = blockIdx.z * kBpZ;
    const bool active = i < g.nx && j < g.ny && kz0 < g.nz;
    const int nzt = FULL ? kBpZ : max(min(kBpZ, g.nz - kz0), 0);  // FULL: nz is a multiple of kBpZ
    // voxel centre relative to the block corner p0 (exact for grid steps)
    const float rx0 = ((float)(i - i0) + 0.5f) * g.dx;
    const float ry0 = ((float)(j - j0) + 0.5f) * g.dy;
    const float rz0 = 0.5f * g.dz;
    const float qx = fmaf((float)i, g.dx, g.bx + 0.5f * g.dx);
    const float qy = fmaf((float)j, g.dy, g.by + 0.5f * g.dy);
    const float qz0 = fmaf((float)kz0, g.dz, g.bz + 0.5f * g.dz);
    const float hx = 0.5f * g.dx, hy = 0.5f * g.dy, hz = 0.5f * g.dz;
    // block corner (FP64), for the re-based maps
    const double p0x = (double)g.bx + (double)i0 * g.dx, p0y = (double)g.by + (double)j0 * g.dy;
    const double p0z = (double)g.bz + (double)kz0 * g.dz;
    float temp[kBpZ], wsum[kBpZ];
#pragma unroll
    for (int t = 0; t < kBpZ; ++t) {
        temp[t] = 0.f;
        wsum[t] = 0.f;
    }
    for (int64_t p = 0; p < nproj; ++p) {
        // one thread re-bases the map to the block, with the pixel origin the
        // TMA-staged kernel gives a block of the same shape (the lowest row /
        // column its 8 corners reach), so both compute the same numbers
        if (tid == 0) {
            const BddProj P = pj[p];
            float umin = 3.4e38f, vmin = 3.4e38f;
            for (int q = 0; q < 8; ++q) {
                const float cx = g.bx + (float)((q & 1) ? min(i0 + (int)blockDim.x, g.nx) : i0) * g.dx;
                const float cy = g.by + (float)((q & 2) ? min(j0 + (int)blockDim.y, g.ny) : j0) * g.dy;
                const float cz = g.bz + (float)((q & 4) ? min(kz0 + kBpZ, g.nz) : kz0) * g.dz;
                const float2 uv = bdd_corner_uv(P, cx, cy, cz);
                umin = fminf(umin, uv.x);
                vmin = fminf(vmin, uv.y);
            }
            const int2 org = bdd_block_origin(umin, vmin, nr, nc);
            bdd_rebase(smap[p & 1], pm[p], P, p0x, p0y, p0z, org.x, org.y);
        }
        __syncthreads();
        if (!active) continue;
        const BddMapR M = smap[p & 1];
        BpFootprint F;
        if (!bdd_bp_footprint(M, rx0, ry0, rz0, hx, hy, hz, qx, qy, g, nr, nc, nzt, F)) continue;
        const Seg &seg = F.seg;
        const int r0 = F.r0, cA = F.cA, ncols = F.ncols;
        const float V0 = F.V0, vl0 = F.vl0, vr0 = F.vr0, svl = F.svl, svr = F.svr;
        const float axy = F.axy, kscale = F.kscale;
        const float *yp = y + p * (int64_t)nr * nc + (int64_t)M.o.y * nr + M.o.x + r0;
#define col_sum(c) seg_sum(seg, yp + (int64_t)(c) * nr)
        if (ncols <= kBpCols) {
            float acc = 0.f;
#pragma unroll
            for (int m = 0; m < kBpCols; ++m) {
                if (m >= ncols) break;
                const float rs = col_sum(cA + m);
                pref[m][tid] = bp_prefix_node(acc, rs, m);
                acc += rs;
            }
            bp_voxels<kBpZ, SENS, FULL, kBpThreads>(F, &pref[0][tid], nzt, nc, qz0 - M.s.z, g.dz, temp, wsum);
        } else {
            // footprints wider than the slot array: per voxel, walk its columns
#pragma unroll
            for (int t = 0; t < kBpZ; ++t) {
                const float vlt = fmaf((float)t, svl, vl0), vrt = fmaf((float)t, svr, vr0);
                const float va = fmaxf(fminf(vlt, vrt), -V0), vb = fminf(fmaxf(vlt, vrt), (float)nc - V0);
                if ((FULL || t < nzt) && vb > va) {
                    const int c0 = (int)floorf(va), c1 = min((int)ceilf(vb), nc - M.o.y) - 1;
                    float apu = 0.f;
                    for (int c = c0; c <= c1; ++c) {
                        const float ov = fminf(vb, (float)(c + 1)) - fmaxf(va, (float)c);
                        apu = fmaf(ov, col_sum(c), apu);
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
#undef col_sum
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

// rows: warps per block (blocks of 32 x rows threads)
template <int C>
static void launch_fp(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                      int64_t nproj, const float *img, const float *imgT, float *y, int rows, cudaStream_t st) {
    const int groups = (nc + C - 1) / C;
    dim3 block(32, rows);
    dim3 grid((nr + 31) / 32, (groups + rows - 1) / rows, (unsigned)nproj);
    k_bdd_fp<C><<<grid, block, 0, st>>>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y);
}

template <int Z, int T>
static void launch_bp_t(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj,
                        const float *y, float *img, float *sens, cudaStream_t st) {
    dim3 block(32, T / 32);
    dim3 grid((g.nx + 31) / 32, (g.ny + block.y - 1) / block.y, (g.nz + Z - 1) / Z);
    const bool full = g.nz % Z == 0;
    if (sens && full)
        k_bdd_bp<Z, true, true, T><<<grid, block, 0, st>>>(g, pj, pm, nr, nc, nproj, y, img, sens);
    else if (sens)
        k_bdd_bp<Z, true, false, T><<<grid, block, 0, st>>>(g, pj, pm, nr, nc, nproj, y, img, sens);
    else if (full)
        k_bdd_bp<Z, false, true, T><<<grid, block, 0, st>>>(g, pj, pm, nr, nc, nproj, y, img, sens);
    else
        k_bdd_bp<Z, false, false, T><<<grid, block, 0, st>>>(g, pj, pm, nr, nc, nproj, y, img, sens);
}

template <int Z>
static void launch_bp(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj,
                      const float *y, float *img, float *sens, int rows, cudaStream_t st) {
    // 16 voxels along z: the prefix slots of 256 threads would exceed 48 KB
    // of static shared memory, so that shape runs 128-thread blocks
    if (rows == 4 || Z == 16)
        launch_bp_t<Z, 128>(g, pj, pm, nr, nc, nproj, y, img, sens, st);
    else
        launch_bp_t<Z < 16 ? Z : 8, 256>(g, pj, pm, nr, nc, nproj, y, img, sens, st);
}

int bdd_forward(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                int64_t nproj, const float *img, float *imgT, float *y, const Tuning &tn, cudaStream_t st) {
    if (nproj <= 0) return OMB_OK;
    if (nproj > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 projections in one call");
    dim3 tg((g.nx + 31) / 32, (g.ny + 31) / 32, g.nz);
    k_transpose_xy<<<tg, dim3(32, 8), 0, st>>>(img, imgT, g.nx, g.ny, g.nz);
    OMB_LAUNCH_CHECK("transpose launch");
    if (tn.bdd_fp_staged && (tn.bdd_fp_cols == 8 || tn.bdd_fp_cols == 16) && bdd_fp_tma_supported(g, img, imgT))
        return bdd_forward_tma(g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y, tn.bdd_fp_cols, st);
    switch (tn.bdd_fp_cols) {
        case 16: launch_fp<16>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y, tn.bdd_fp_rows, st); break;
        default: launch_fp<8>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y, tn.bdd_fp_rows, st); break;
    }
    OMB_LAUNCH_CHECK("bdd forward launch");
    return OMB_OK;
}

int bdd_backward_ray(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                     int64_t nproj, const float *y, float *img, float *sens, unsigned long long *acc,
                     unsigned long long *acc_s, cudaStream_t st) {
    if (nproj <= 0) return OMB_OK;
    if (nproj > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 projections in one call");
    const int groups = (nc + 7) / 8;
    dim3 block(32, 4);
    dim3 grid((nr + 31) / 32, (groups + 3) / 4, (unsigned)nproj);
    if (acc) {
        if (acc_s)
            k_bdd_bp_ray<true, true><<<grid, block, 0, st>>>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, y, img, sens,
                                                              acc, acc_s);
        else
            k_bdd_bp_ray<true, false><<<grid, block, 0, st>>>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, y, img, sens,
                                                               acc, acc_s);
    } else if (sens) {
        k_bdd_bp_ray<false, true><<<grid, block, 0, st>>>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, y, img, sens,
                                                           acc, acc_s);
    } else {
        k_bdd_bp_ray<false, false><<<grid, block, 0, st>>>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, y, img, sens,
                                                            acc, acc_s);
    }
    OMB_LAUNCH_CHECK("type-5 ray-driven backward launch");
    return OMB_OK;
}

int bdd_backward(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj, const float *y,
                 float *img, float *sens, const Tuning &tn, cudaStream_t st) {
    if (g.nz > 65535 * 4) return set_error(OMB_ERR_UNSUPPORTED, "too many slices");
    if (tn.bdd_bp_staged && (tn.bdd_bp_z == 8 || tn.bdd_bp_z == 16) && bdd_bp_tma_supported(nr, y))
        return bdd_backward_tma(g, pj, pm, nr, nc, nproj, y, img, sens, tn.bdd_bp_z, st);
    const int rows = tn.bdd_bp_rows;
    switch (tn.bdd_bp_z) {
        case 4: launch_bp<4>(g, pj, pm, nr, nc, nproj, y, img, sens, rows, st); break;
        case 16: launch_bp<16>(g, pj, pm, nr, nc, nproj, y, img, sens, rows, st); break;
        default: launch_bp<8>(g, pj, pm, nr, nc, nproj, y, img, sens, rows, st); break;
    }
    OMB_LAUNCH_CHECK("bdd backward launch");
    return OMB_OK;
}

}  // namespace omb
