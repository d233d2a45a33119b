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
#include "kernels.h"

namespace omb {

constexpr int kColsPerThread = 8;

// Per-ray constants of the forward projection: footprint edge lines in voxel
// units, e(j) = e0 + j * e1 for slice j, and the pixel's weight.
struct BddRay {
    float xa0, xa1, xb0, xb1;   // lateral edges (voxel units of the in-slice axis)
    float dw0, dw1;             // lateral width  xb - xa (for the area)
    float za0, za1, zb0, zb1;   // axial edges (voxel units of z), first column
    float dz0, dz1;             // axial width zb - za
    float kerroin;              // dx*dy*dz / |u_axis|
    bool ysl;                   // slices along y (|s.x| <= |s.y|)
};

__device__ __forceinline__ BddRay bdd_ray_setup(const Grid &g, const float *__restrict__ xy,
                                                const float *__restrict__ uv, int64_t gp, int r, int c0, int nr,
                                                int nc, float pitch_y) {
    const float *q = xy + gp * 6;
    const double sx = __ldg(q), sy = __ldg(q + 1), sz = __ldg(q + 2);
    const double cx = __ldg(q + 3), cy = __ldg(q + 4), cz = __ldg(q + 5);
    const double ux = __ldg(uv + gp * 2), uy = __ldg(uv + gp * 2 + 1);
    const double ia = (double)r - (double)nr / 2.0 + 0.5;
    const double ib = (double)c0 - (double)nc / 2.0 + 0.5;
    const double dx = cx + ia * ux, dy = cy + ia * uy, dz = cz + ib * (double)pitch_y;
    const double dLx = dx + 0.5 * ux, dLy = dy + 0.5 * uy;   // dL
    const double dRx = dx - 0.5 * ux, dRy = dy - 0.5 * uy;   // dR
    const double dUz = dz + 0.5 * (double)pitch_y, dDz = dz - 0.5 * (double)pitch_y;
    const double vx = dx - sx, vy = dy - sy, vz = dz - sz;
    const double L = sqrt(vx * vx + vy * vy + vz * vz);
    const double gdx = g.dx, gdy = g.dy, gdz = g.dz;
    BddRay b;
    b.ysl = fabs(sx) <= fabs(sy);
    double kerroin = gdx * gdy * gdz;
    const double zoff = (double)g.bz - sz;  // z of the slice origin relative to the source
    double a0, a1, c0v, c1v, step, base, lat_off, lat_d;
    if (b.ysl) {
        a0 = (dLx - sx) / (dLy - sy);
        a1 = (dRx - sx) / (dRy - sy);
        c0v = (dUz - sz) / (dy - sy);
        c1v = (dDz - sz) / (dy - sy);
        kerroin /= fabs(vy / L);
        base = (double)g.by - sy + 0.5 * gdy;   // v of slice 0 (its centre)
        step = gdy;
        lat_off = (double)g.bx - sx;            // lateral origin relative to the source
        lat_d = gdx;
    } else {
        a0 = (dLy - sy) / (dLx - sx);
        a1 = (dRy - sy) / (dRx - sx);
        c0v = (dUz - sz) / (dx - sx);
        c1v = (dDz - sz) / (dx - sx);
        kerroin /= fabs(vx / L);
        base = (double)g.bx - sx + 0.5 * gdx;
        step = gdx;
        lat_off = (double)g.by - sy;
        lat_d = gdy;
    }
    // edge (in voxel units from the grid corner) on slice j: (v_j * slope - off) / d
    b.xa0 = (float)((base * a0 - lat_off) / lat_d);
    b.xa1 = (float)(step * a0 / lat_d);
    b.xb0 = (float)((base * a1 - lat_off) / lat_d);
    b.xb1 = (float)(step * a1 / lat_d);
    b.dw0 = (float)(base * (a1 - a0) / lat_d);
    b.dw1 = (float)(step * (a1 - a0) / lat_d);
    b.za0 = (float)((base * c0v - zoff) / gdz);
    b.za1 = (float)(step * c0v / gdz);
    b.zb0 = (float)((base * c1v - zoff) / gdz);
    b.zb1 = (float)(step * c1v / gdz);
    b.dz0 = (float)(base * (c1v - c0v) / gdz);
    b.dz1 = (float)(step * (c1v - c0v) / gdz);
    b.kerroin = (float)kerroin;
    return b;
}

// Forward projection.  Thread = (detector row, group of 8 columns, projection).
// `img` is x-fastest, `imgT` the same image y-fastest; slices along y read
// `img`, slices along x read `imgT`, so a warp's 32 rows read consecutive
// addresses in both cases.
__global__ void __launch_bounds__(256) k_bdd_fp(Grid g, const float *__restrict__ xy, const float *__restrict__ uv,
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
    const int nsl = b.ysl ? g.ny : g.nx;       // slices
    const int nlat = b.ysl ? g.nx : g.ny;      // voxels across a slice
    const int64_t lat_stride = 1;              // both layouts: lateral axis fastest
    const int64_t sl_stride = nlat;
    const int64_t z_stride = (int64_t)g.nx * g.ny;
    const float *__restrict__ vol = b.ysl ? img : imgT;
    const float flat = (float)nlat, fz = (float)g.nz;
    const float dlat = b.ysl ? g.dx : g.dy;
    float temp[kColsPerThread];
#pragma unroll
    for (int c = 0; c < kColsPerThread; ++c) temp[c] = 0.f;

    for (int j = 0; j < nsl; ++j) {
        const float fj = (float)j;
        float xa = fmaf(fj, b.xa1, b.xa0), xb = fmaf(fj, b.xb1, b.xb0);
        float za = fmaf(fj, b.za1, b.za0), zb = fmaf(fj, b.zb1, b.zb0);
        const float el = fminf(xa, xb), er = fmaxf(xa, xb);
        const float zu = fminf(za, zb);
        const float w = fabsf(fmaf(fj, b.dz1, b.dz0));
        const float area = fabsf(fmaf(fj, b.dw1, b.dw0)) * dlat * w * g.dz;
        const float inv_area = 1.f / area;
        // lateral overlap range (clamped to the slice)
        const float cl = fmaxf(el, 0.f), cr = fminf(er, flat);
        if (!(cr > cl)) continue;
        const int i0 = (int)floorf(cl);
        const int i1 = min((int)ceilf(cr), nlat) - 1;
        // axial range of all columns: [zu, zu + ncol*w]
        const float zl_all = fmaxf(zu, 0.f), zr_all = fminf(fmaf((float)ncol, w, zu), fz);
        if (!(zr_all > zl_all)) continue;
        const int k0 = (int)floorf(zl_all);
        const int k1 = min((int)ceilf(zr_all), g.nz) - 1;
        const float *slice = vol + (int64_t)j * sl_stride;
        for (int k = k0; k <= k1; ++k) {
            // lateral integral of row (slice j, z k) over the footprint
            const float *row = slice + (int64_t)k * z_stride;
            float rk = 0.f;
            for (int i = i0; i <= i1; ++i) {
                const float ox = fminf(cr, (float)(i + 1)) - fmaxf(cl, (float)i);
                rk = fmaf(ox, __ldg(row + i * lat_stride), rk);
            }
            if (rk == 0.f) continue;
            const float kl = (float)k, kr = (float)(k + 1);
#pragma unroll
            for (int c = 0; c < kColsPerThread; ++c) {
                const float lo = fmaf((float)c, w, zu), hi = fmaf((float)(c + 1), w, zu);
                const float oz = fminf(hi, kr) - fmaxf(lo, kl);
                if (c < ncol && oz > 0.f) temp[c] = fmaf(rk * oz, inv_area, temp[c]);
            }
        }
    }
    int64_t idx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
#pragma unroll
    for (int c = 0; c < kColsPerThread; ++c)
        if (c < ncol) y[idx + (int64_t)c * nr] = temp[c] * b.kerroin;
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

__global__ void __launch_bounds__(256) k_bdd_bp(Grid g, const BddProj *__restrict__ pj, int nr, int nc,
                                                int64_t nproj, const float *__restrict__ y,
                                                float *__restrict__ img, float *__restrict__ sens) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    const float qx = fmaf((float)i, g.dx, g.bx + 0.5f * g.dx);
    const float qy = fmaf((float)j, g.dy, g.by + 0.5f * g.dy);
    const float qz = fmaf((float)k, g.dz, g.bz + 0.5f * g.dz);
    const float hx = 0.5f * g.dx, hy = 0.5f * g.dy, hz = 0.5f * g.dz;
    const float fnr = (float)nr, fnc = (float)nc;
    float temp = 0.f, wsum = 0.f;
    for (int64_t p = 0; p < nproj; ++p) {
        const BddProj P = pj[p];
        // mid-plane corners LU and RD of the voxel (projectorType5.cl:508-527)
        float lx, ly, rx, ry;
        if (P.ysl) {
            const float sgn = P.spos ? 1.f : -1.f;
            lx = qx - sgn * hx; rx = qx + sgn * hx; ly = qy; ry = qy;
        } else {
            const float sgn = P.spos ? 1.f : -1.f;
            lx = qx; rx = qx; ly = qy + sgn * hy; ry = qy - sgn * hy;
        }
        const float lz = qz - hz, rz = qz + hz;
        const float dl = 1.f / fmaf(P.c[0], lx, fmaf(P.c[1], ly, fmaf(P.c[2], lz, 1.f)));
        const float dr = 1.f / fmaf(P.c[0], rx, fmaf(P.c[1], ry, fmaf(P.c[2], rz, 1.f)));
        const float ul = fmaf(P.au[0], lx, fmaf(P.au[1], ly, fmaf(P.au[2], lz, P.au0))) * dl;
        const float ur = fmaf(P.au[0], rx, fmaf(P.au[1], ry, fmaf(P.au[2], rz, P.au0))) * dr;
        const float vl = fmaf(P.av[0], lx, fmaf(P.av[1], ly, fmaf(P.av[2], lz, P.av0))) * dl;
        const float vr = fmaf(P.av[0], rx, fmaf(P.av[1], ry, fmaf(P.av[2], rz, P.av0))) * dr;
        const float ua = fmaxf(fminf(ul, ur), 0.f), ub = fminf(fmaxf(ul, ur), fnr);
        const float va = fmaxf(fminf(vl, vr), 0.f), vb = fminf(fmaxf(vl, vr), fnc);
        if (!(ub > ua) || !(vb > va)) continue;
        const int r0 = (int)floorf(ua), r1 = min((int)ceilf(ub), nr) - 1;
        const int c0 = (int)floorf(va), c1 = min((int)ceilf(vb), nc) - 1;
        const float *yp = y + p * (int64_t)nr * nc;
        float apu = 0.f;
        for (int c = c0; c <= c1; ++c) {
            const float ov = fminf(vb, (float)(c + 1)) - fmaxf(va, (float)c);
            float row = 0.f;
            for (int rr = r0; rr <= r1; ++rr) {
                const float ou = fminf(ub, (float)(rr + 1)) - fmaxf(ua, (float)rr);
                row = fmaf(ou, __ldg(yp + rr + (int64_t)c * nr), row);
            }
            apu = fmaf(ov, row, apu);
        }
        if (apu != 0.f) {
            // d * |v| / |v_axis| with v = voxel centre - source
            const float vx = qx - P.s[0], vy = qy - P.s[1], vz = qz - P.s[2];
            const float len = sqrtf(vx * vx + vy * vy + vz * vz);
            const float ker = P.ysl ? g.dy * len / fabsf(vy) : g.dx * len / fabsf(vx);
            temp = fmaf(apu, ker, temp);
            wsum += ker;
        }
    }
    const int64_t n = i + (int64_t)j * g.nx + (int64_t)k * g.nx * g.ny;
    img[n] = temp;
    if (sens) sens[n] = wsum;
}

int bdd_forward(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                int64_t nproj, const float *img, float *imgT, float *y, cudaStream_t st) {
    if (nproj <= 0) return OMB_OK;
    if (nproj > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 projections in one call");
    dim3 tg((g.nx + 31) / 32, (g.ny + 31) / 32, g.nz);
    k_transpose_xy<<<tg, dim3(32, 8), 0, st>>>(img, imgT, g.nx, g.ny, g.nz);
    OMB_LAUNCH_CHECK("transpose launch");
    const int groups = (nc + kColsPerThread - 1) / kColsPerThread;
    dim3 block(32, 8);
    dim3 grid((nr + 31) / 32, (groups + 7) / 8, (unsigned)nproj);
    k_bdd_fp<<<grid, block, 0, st>>>(g, xy, uv, nr, nc, pitch_y, proj0, nproj, img, imgT, y);
    OMB_LAUNCH_CHECK("bdd forward launch");
    return OMB_OK;
}

int bdd_backward(const Grid &g, const BddProj *pj, int nr, int nc, int64_t nproj, const float *y, float *img,
                 float *sens, cudaStream_t st) {
    if (g.nz > 65535) return set_error(OMB_ERR_UNSUPPORTED, "more than 65535 slices");
    dim3 block(32, 8);
    dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
    k_bdd_bp<<<grid, block, 0, st>>>(g, pj, nr, nc, nproj, y, img, sens);
    OMB_LAUNCH_CHECK("bdd backward launch");
    return OMB_OK;
}

}  // namespace omb
