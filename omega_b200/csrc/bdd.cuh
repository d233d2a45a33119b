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

// Slices [lo, hi] outside which a group of rays cannot meet the volume: a
// forward-projection thread (one ray group) or a CTA (the union of its
// corner ray groups) loops over these slices only.  The slices where a ray
// group's footprint meets the volume satisfy four conditions, each the union
// of half-lines in j (the footprint edges are linear in the slice index):
//   lateral  min(xa, xb) < nlat  and  max(xa, xb) > 0,
//   axial    min(za, zb) < nz    and  the group's top > 0, where the top of
//            C columns is zu + C|zb - za|, bounded by C zb - (C-1) za or
//            C za - (C-1) zb.
// Each condition's solution set is replaced by the hull of its half-lines
// (one slice of margin at each end) and the hulls are intersected: a superset
// of the true slices, so skipping the others changes no result -- outside
// them every column's footprint integral is exactly zero.
struct SliceHull {
    int lo, hi;  // hull of the half-lines added so far; lo > hi: empty
};

// adds {j in [0, nsl-1] : a + b j > c} to the hull
__device__ __forceinline__ void slice_halfline(SliceHull &h, float a, float b, float c, int nsl) {
    int lo = 0, hi = nsl - 1;
    if (fabsf(b) * (float)nsl <= 1e-6f * (fabsf(a) + fabsf(c) + 1.f)) {
        if (!(a > c - 1e-4f * (fabsf(c) + 1.f))) return;  // constant and false
    } else {
        const float js = (c - a) / b;
        if (b > 0.f) {
            if (js >= (float)nsl) return;
            lo = max((int)floorf(js) - 1, 0);
        } else {
            if (js < 0.f) return;
            hi = min((int)ceilf(js) + 1, nsl - 1);
        }
    }
    if (lo > hi) return;
    h.lo = min(h.lo, lo);
    h.hi = max(h.hi, hi);
}

// The four condition hulls of one ray group (edges e(j) = e0 + j e1 in voxel
// units, as BddRay holds them), accumulated over several groups.
struct SliceRange {
    SliceHull lat_lo, lat_hi, ax_lo, ax_hi;
};

__device__ __forceinline__ SliceRange slice_range_empty() {
    SliceRange r;
    r.lat_lo = r.lat_hi = r.ax_lo = r.ax_hi = SliceHull{1 << 30, -1};
    return r;
}

__device__ __forceinline__ void slice_range_add(SliceRange &r, float xa0, float xa1, float xb0, float xb1, float za0,
                                                float za1, float zb0, float zb1, int nsl, int nlat, int nz,
                                                float C) {
    slice_halfline(r.lat_lo, -xa0, -xa1, -(float)nlat, nsl);
    slice_halfline(r.lat_lo, -xb0, -xb1, -(float)nlat, nsl);
    slice_halfline(r.lat_hi, xa0, xa1, 0.f, nsl);
    slice_halfline(r.lat_hi, xb0, xb1, 0.f, nsl);
    slice_halfline(r.ax_lo, -za0, -za1, -(float)nz, nsl);
    slice_halfline(r.ax_lo, -zb0, -zb1, -(float)nz, nsl);
    slice_halfline(r.ax_hi, C * zb0 - (C - 1.f) * za0, C * zb1 - (C - 1.f) * za1, 0.f, nsl);
    slice_halfline(r.ax_hi, C * za0 - (C - 1.f) * zb0, C * za1 - (C - 1.f) * zb1, 0.f, nsl);
}

// [lo, hi] of the slices to visit (lo > hi: none)
__device__ __forceinline__ int2 slice_range_bounds(const SliceRange &r) {
    return make_int2(max(max(r.lat_lo.lo, r.lat_hi.lo), max(r.ax_lo.lo, r.ax_hi.lo)),
                     min(min(r.lat_lo.hi, r.lat_hi.hi), min(r.ax_lo.hi, r.ax_hi.hi)));
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

// One voxel column's footprint on one projection for the backprojection:
// rows [ua, ub] (shared by the column's voxels: u does not depend on z for
// these panels) with their weights `seg`, the columns [vA, vB] the whole run
// of nzt voxels covers, and the per-voxel column edges v = v0 + t s (left and
// right corner).  Coordinates are relative to the re-based map's pixel origin
// (U0, V0); (rx0, ry0, rz0) is the first voxel's centre relative to the
// block corner, (qx, qy) its world x and y.  False when the footprint misses
// the panel.
struct BpFootprint {
    Seg seg;
    int r0, cA, ncols;
    float U0, V0;
    float vl0, vr0, svl, svr, vmin, vmax, vA, vB;
    float axy, kscale;
};

__device__ __forceinline__ bool bdd_bp_footprint(const BddMapR &M, float rx0, float ry0, float rz0, float hx, float hy,
                                                 float hz, float qx, float qy, const Grid &g, int nr, int nc, int nzt,
                                                 BpFootprint &F) {
    F.U0 = M.s.w;
    F.V0 = (float)M.o.y;
    float lx, ly, rx, ry;
    const float sgn = M.o.w ? 1.f : -1.f;
    if (M.o.z) {
        lx = rx0 - sgn * hx; rx = rx0 + sgn * hx; ly = ry0; ry = ry0;
    } else {
        lx = rx0; rx = rx0; ly = ry0 + sgn * hy; ry = ry0 - sgn * hy;
    }
    const float dl = 1.f / fmaf(M.c.x, lx, fmaf(M.c.y, ly, fmaf(M.c.z, rz0, M.c.w)));
    const float dr = 1.f / fmaf(M.c.x, rx, fmaf(M.c.y, ry, fmaf(M.c.z, rz0, M.c.w)));
    const float ul = fmaf(M.u.x, lx, fmaf(M.u.y, ly, fmaf(M.u.z, rz0, M.u.w))) * dl;
    const float ur = fmaf(M.u.x, rx, fmaf(M.u.y, ry, fmaf(M.u.z, rz0, M.u.w))) * dr;
    const float ua = fmaxf(fminf(ul, ur), -F.U0), ub = fminf(fmaxf(ul, ur), (float)nr - F.U0);
    if (!(ub > ua)) return false;
    F.r0 = (int)floorf(ua);
    F.seg = make_seg(ua, ub, F.r0, min((int)ceilf(ub), nr - M.o.x) - 1 - F.r0);
    F.vl0 = fmaf(M.v.x, lx, fmaf(M.v.y, ly, fmaf(M.v.z, rz0 - hz, M.v.w))) * dl;
    F.vr0 = fmaf(M.v.x, rx, fmaf(M.v.y, ry, fmaf(M.v.z, rz0 + hz, M.v.w))) * dr;
    F.svl = M.v.z * g.dz * dl;
    F.svr = M.v.z * g.dz * dr;
    const float tl = (float)(nzt - 1);
    F.vmin = fminf(fminf(F.vl0, F.vr0), fminf(fmaf(tl, F.svl, F.vl0), fmaf(tl, F.svr, F.vr0)));
    F.vmax = fmaxf(fmaxf(F.vl0, F.vr0), fmaxf(fmaf(tl, F.svl, F.vl0), fmaf(tl, F.svr, F.vr0)));
    F.vA = fmaxf(F.vmin, -F.V0);
    F.vB = fminf(F.vmax, (float)nc - F.V0);
    if (!(F.vB > F.vA)) return false;
    // kerroin = d * |v| / |v_axis|, v = voxel centre - source
    const float vx = qx - M.s.x, vy = qy - M.s.y;
    F.axy = vx * vx + vy * vy;
    F.kscale = M.o.z ? __fdividef(g.dy, fabsf(vy)) : __fdividef(g.dx, fabsf(vx));
    F.cA = (int)floorf(F.vA);
    F.ncols = min((int)ceilf(F.vB), nc - M.o.y) - F.cA;
    return true;
}

// Node m of a column prefix: the prefix P(x) = (sum of the row sums of the
// columns before m) + (x - m) rs_m for x in [m, m + 1] (x relative to the
// first column), stored as its intercept and slope, P(x) = B_m + x rs_m.
__device__ __forceinline__ float2 bp_prefix_node(float acc, float rs, int m) {
    return make_float2(fmaf(-(float)m, rs, acc), rs);
}

// The voxels of one column on one projection, from the prefix nodes
// pc[m * STRIDE] (bp_prefix_node), m < ncols: voxel t covers the detector
// columns between its edges a_t = vl0 + t svl and b_t = vr0 + t svr
// (relative to column cA, as fractional column positions), and its value is
// the prefix difference P(max) - P(min).  IN: every edge lies on the panel
// (no clamp to [vA, vB]); CR: the two edge lines cross inside the run (the
// lower edge is taken per voxel).  Shared by the staged and unstaged kernels,
// which therefore compute the same numbers.
template <int KZ, bool SENS, bool FULL, int STRIDE, bool IN, bool CR>
__device__ __forceinline__ void bp_voxel_run(const float2 *__restrict__ pc, int nzt, int mmax, float a0, float sa,
                                             float b0, float sb, float vAr, float vBr, float vz0, float dz, float axy,
                                             float kscale, float *temp, float *wsum) {
#pragma unroll
    for (int t = 0; t < KZ; ++t) {
        if (FULL || t < nzt) {
            const float at = fmaf((float)t, sa, a0), bt = fmaf((float)t, sb, b0);
            float lo = CR ? fminf(at, bt) : at, hi = CR ? fmaxf(at, bt) : bt;
            if (!IN) {
                lo = fminf(fmaxf(lo, vAr), vBr);
                hi = fminf(fmaxf(hi, vAr), vBr);
            }
            const int ma = min((int)lo, mmax), mb = min((int)hi, mmax);
            const float2 ea = pc[ma * STRIDE], eb = pc[mb * STRIDE];
            const float apu = fmaf(hi, eb.y, eb.x) - fmaf(lo, ea.y, ea.x);
            if (SENS) {
                if (apu != 0.f) {
                    const float vz = fmaf((float)t, dz, vz0);
                    const float q2 = fmaf(vz, vz, axy);
                    const float ker = kscale * (q2 * rsqrtf(q2));
                    temp[t] = fmaf(apu, ker, temp[t]);
                    wsum[t] += ker;
                }
            } else {
                // branch-free: with apu = 0 the multiply-add leaves the sum as it is (q2 >= axy > 0, so ker
                // is finite)
                const float vz = fmaf((float)t, dz, vz0);
                const float q2 = fmaf(vz, vz, axy);
                temp[t] = fmaf(apu, kscale * (q2 * rsqrtf(q2)), temp[t]);
            }
        }
    }
}

template <int KZ, bool SENS, bool FULL, int STRIDE>
__device__ __forceinline__ void bp_voxels(const BpFootprint &F, const float2 *__restrict__ pc, int nzt, int nc,
                                          float vz0, float dz, float *temp, float *wsum) {
    const float fA = (float)F.cA;
    const int mmax = F.ncols - 1;
    float a0 = F.vl0 - fA, b0 = F.vr0 - fA, sa = F.svl, sb = F.svr;
    const float tl = (float)((FULL ? KZ : nzt) - 1);
    const float aL = fmaf(tl, sa, a0), bL = fmaf(tl, sb, b0);
    const bool cross = (a0 <= b0) != (aL <= bL);
    if (!cross && b0 < a0) {
        // the right-corner edge is the lower one throughout
        float u = a0;
        a0 = b0;
        b0 = u;
        u = sa;
        sa = sb;
        sb = u;
    }
    const bool in = F.vmin >= -F.V0 && F.vmax <= (float)nc - F.V0;
    const float vAr = F.vA - fA, vBr = F.vB - fA;
    if (!cross) {
        if (in)
            bp_voxel_run<KZ, SENS, FULL, STRIDE, true, false>(pc, nzt, mmax, a0, sa, b0, sb, vAr, vBr, vz0, dz, F.axy,
                                                             F.kscale, temp, wsum);
        else
            bp_voxel_run<KZ, SENS, FULL, STRIDE, false, false>(pc, nzt, mmax, a0, sa, b0, sb, vAr, vBr, vz0, dz,
                                                              F.axy, F.kscale, temp, wsum);
    } else {
        bp_voxel_run<KZ, SENS, FULL, STRIDE, false, true>(pc, nzt, mmax, a0, sa, b0, sb, vAr, vBr, vz0, dz, F.axy,
                                                         F.kscale, temp, wsum);
    }
}

// seg_sum over a run staged in shared memory (plain loads, same arithmetic).
__device__ __forceinline__ float seg_sum_shared(const Seg &s, const float *p) {
    float acc = fmaf(s.w2, p[s.o2], fmaf(s.w1, p[s.o1], s.w0 * p[0]));
    for (int i = 3; i <= s.n; ++i) acc = fmaf(fminf(s.hi, (float)(s.base + i + 1)) - (float)(s.base + i), p[i], acc);
    return acc;
}

}  // namespace omb
