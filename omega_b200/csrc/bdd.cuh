// Shared device helpers of the type-5 (branchless distance-driven)
// projectors: the forward projection's per-ray footprint lines and the
// weighted sums over a run of voxels or detector pixels.
#pragma once
#include "common.cuh"

namespace omb {

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

// The forward weight dx*dy*dz / |u_axis| of the ray through pixel (r, c).
__device__ __forceinline__ float bdd_kerroin(const Grid &g, const float *__restrict__ xy,
                                             const float *__restrict__ uv, int64_t gp, int r, int c, int nr, int nc,
                                             float pitch_y, bool ysl) {
    const float *q = xy + gp * 6;
    const double sx = __ldg(q), sy = __ldg(q + 1), sz = __ldg(q + 2);
    const double ux = __ldg(uv + gp * 2), uy = __ldg(uv + gp * 2 + 1);
    const double ia = (double)r - (double)nr / 2.0 + 0.5;
    const double ib = (double)c - (double)nc / 2.0 + 0.5;
    const double vx = __ldg(q + 3) + ia * ux - sx, vy = __ldg(q + 4) + ia * uy - sy;
    const double vz = __ldg(q + 5) + ib * (double)pitch_y - sz;
    const double L = sqrt(vx * vx + vy * vy + vz * vz);
    return (float)((double)g.dx * g.dy * g.dz / fabs((ysl ? vy : vx) / L));
}

// Weighted sum along one contiguous run of voxels / detector pixels that
// overlap [lo, hi]: element 0 (at `base`, lo >= base) partial, then full
// elements, the last one partial again.  Up to three elements take a fixed
// three-load path with zero weights for the missing ones (index clamped).
struct Seg {
    float w0, w1, w2, hi;
    int o1, o2, n, base;
};

__device__ __forceinline__ Seg make_seg(float lo, float hi, int base, int n) {
    Seg s;
    s.hi = hi;
    s.base = base;
    s.n = n;
    s.w0 = fminf(hi, (float)(base + 1)) - lo;
    s.w1 = n == 0 ? 0.f : (n == 1 ? hi - (float)(base + 1) : 1.f);
    s.w2 = n < 2 ? 0.f : (n == 2 ? hi - (float)(base + 2) : 1.f);
    s.o1 = min(n, 1);
    s.o2 = min(n, 2);
    return s;
}

__device__ __forceinline__ float seg_sum(const Seg &s, const float *__restrict__ p) {
    float acc = fmaf(s.w2, __ldg(p + s.o2), fmaf(s.w1, __ldg(p + s.o1), s.w0 * __ldg(p)));
    for (int i = 3; i <= s.n; ++i)
        acc = fmaf(fminf(s.hi, (float)(s.base + i + 1)) - (float)(s.base + i), __ldg(p + i), acc);
    return acc;
}

// detector columns one thread's run of kBpZ voxels may cover before it takes
// the per-voxel path (about 1.25 columns per voxel at magnification 2)
__host__ __device__ constexpr int bp_slots(int kBpZ) { return kBpZ + kBpZ / 2 + (kBpZ < 16 ? 4 : 0); }

// seg_sum over a run staged in shared memory (plain loads, same arithmetic).
__device__ __forceinline__ float seg_sum_shared(const Seg &s, const float *p) {
    float acc = fmaf(s.w2, p[s.o2], fmaf(s.w1, p[s.o1], s.w0 * p[0]));
    for (int i = 3; i <= s.n; ++i) acc = fmaf(fminf(s.hi, (float)(s.base + i + 1)) - (float)(s.base + i), p[i], acc);
    return acc;
}

}  // namespace omb
