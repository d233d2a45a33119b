// Projector types 2 (orthogonal distance) and 3 (volume of intersection),
// PET, forward and backward.
//
// Restates the tube-of-response tracer of OMEGA's projectorType123.cl built
// with -DORTH (-DVOL for type 3) and -DCRYSTXY / -DCRYSTZ: ray set-up
// 493-508 (orth_ray_length = L * width for type 2, L for type 3; TotV =
// L * r^2 / pi), in-plane rows 514-760, oblique rays 791-1296, and
// orthDistance3D / orthogonalHelper3D / compute_element_orth_3D of
// opencl_functions_orth3D.h:24-417.  The ray is walked voxel by voxel as the
// Siddon tracer walks it; every time it leaves a slice through the slice face
// (slices along x, or along y when the ray is closer to the y axis), that
// slice is scanned outward from the ray's voxel -- rows in z up and down,
// columns both ways in each row -- until a voxel centre lies outside the
// tube.  The slices before the ray's first voxel and after its last are
// scanned until one contributes nothing.  Voxel weight: 1 - d / width (type
// 2, cut at 0.01), or the tabulated sphere-cylinder intersection volume at
// distance d (type 3).
//
// Deliberate differences from the reference kernel:
//  * the walk and every distance are FP64 (the reference: FP32), so whether
//    a voxel centre lies inside the tube is decided as the FP64 oracle
//    decides it; weights and TOF are FP32 (the type-3 table index is the
//    FP64 one);
//  * voxel centres are b + (i + 1/2) d each time (the reference steps some of
//    them by repeated addition);
//  * a type-3 table index past its last entry reads the last entry (the
//    reference reads past the table);
//  * a ray that never leaves a slice through its slice face starts the
//    trailing scan as if its last slice had been scanned (the reference's
//    slice marker is uninitialised there; its CPU projector sets it to 0);
//  * TOF along an image row starts at +-half the row with the sign the
//    reference CPU projector takes (copysign of the near-zero transverse
//    component), as the type-1 tracer here does.
// The image must be square transaxially (Nx = Ny, dx = dy, bx = by): the
// reference's in-plane-row branch mixes the x and y counts in its indices.
#include "kernels.h"
#include "siddon.cuh"

namespace omb {
namespace {

constexpr int kBlockO = 128;
constexpr double kThr = 0.01;
constexpr double kCC = 1e3;

struct OrthRay {
    double sx, sy, sz;          // source, slice axis first
    double fx, fy, fz;          // d - s, same order
    double orl;                 // orth_ray_length
    double cut2;                // squared cut-off distance times orl^2: type 2 (1 - 0.01)^2, type 3 bmax^2
    float inv_orl;              // 1 / orl (FP32 weights)
    double b1, d1;              // slice axis
    double b2, d2;              // in-slice axis
    int n1;                     // in-slice count
    int64_t st_slice, st_in, nxy;
};

// orthogonalHelper3D: false = outside the tube (stop the scan), true = visited.
// Whether a voxel is inside is decided on the FP64 squared distance against
// the ray's FP64 cut-off (no square root); the type-2 weight is then formed in
// FP32 (1e-7 relative), the type-3 table index from the FP64 distance, as the
// restatement forms it.
template <class Visit>
__device__ __forceinline__ bool orth_voxel(const Orth &o, const OrthRay &r, int slice, int uu, int zz, double lx,
                                           double ly, double lz, Visit &vis) {
    const double cy = r.b2 + (double)uu * r.d2 + r.d2 * 0.5;
    const double x0 = cy - r.sy;
    const double y1 = r.fz * x0 - ly;
    const double z1 = -r.fx * x0 + lz;
    const double n2 = lx * lx + y1 * y1 + z1 * z1;
    if (o.type == 3 ? n2 > r.cut2 : n2 >= r.cut2) return false;
    float ele;
    if (o.type == 3) {
        const double dd = sqrt(n2) / r.orl;
        ele = dd < (double)o.bmin ? o.vmax : __ldg(o.v + min((int)rint((dd - (double)o.bmin) * kCC), o.nv - 1));
    } else {
        ele = 1.f - sqrtf((float)n2) * r.inv_orl;
    }
    vis((int64_t)slice * r.st_slice + (int64_t)uu * r.st_in + (int64_t)zz * r.nxy, ele);
    return true;
}

// One z row of a slice (the in-slice scans of orthDistance3D).
template <class Visit>
__device__ __forceinline__ void orth_row(const Orth &o, const Grid &g, const OrthRay &r, int slice, int temp2, int zz,
                                         double apu1, double lz, int &uu1, int &uu2, bool &brk, int &count,
                                         Visit &vis) {
    const double cz = (double)g.bz + (double)zz * (double)g.dz + (double)g.dz * 0.5;
    const double z0 = cz - r.sz;
    const double lx = r.fx * z0 - apu1;
    const double ly = r.fy * z0;
    if (!o.xy) {
        uu1 = temp2;
        brk = !orth_voxel(o, r, slice, temp2, zz, lx, ly, lz, vis);
        uu2 = temp2 - 1;
        return;
    }
    for (uu1 = max(temp2, 0); uu1 < r.n1; ++uu1) {
        brk = !orth_voxel(o, r, slice, uu1, zz, lx, ly, lz, vis);
        if (brk) break;
        ++count;
    }
    for (uu2 = min(temp2, r.n1) - 1; uu2 >= 0; --uu2) {
        brk = !orth_voxel(o, r, slice, uu2, zz, lx, ly, lz, vis);
        if (brk) break;
        ++count;
    }
}

// orthDistance3D: scans one slice; returns the number of voxels visited.
template <class Visit>
__device__ int orth_slice(const Orth &o, const Grid &g, const OrthRay &r, int slice, int temp2, int tempk,
                          bool pre_step, int &k, int ku, Visit &vis) {
    int count = 0, uu1 = 0, uu2 = 0, zz;
    bool brk = false;
    const double cx = r.b1 + (double)slice * r.d1 + r.d1 * 0.5;
    const double v0 = cx - r.sx;
    const double lz = r.fy * v0;
    const double apu1 = r.fz * v0;
    if (!o.z) {
        orth_row(o, g, r, slice, temp2, tempk, apu1, lz, uu1, uu2, brk, count, vis);
        return count;
    }
    for (zz = max(tempk, 0); zz < g.nz; ++zz) {
        orth_row(o, g, r, slice, temp2, zz, apu1, lz, uu1, uu2, brk, count, vis);
        if (uu1 == temp2 && uu2 == temp2 - 1 && brk) break;
    }
    k = zz - 1;
    for (zz = min(tempk, g.nz) - 1; zz >= 0; --zz) {
        orth_row(o, g, r, slice, temp2, zz, apu1, lz, uu1, uu2, brk, count, vis);
        if (uu1 == temp2 && uu2 == temp2 - 1 && brk) break;
    }
    if (pre_step) k = ku < 0 ? max(k, zz) - 1 : min(k, zz) + 1;
    return count;
}

// d_g_s / s_g_d in FP64 keeping the first crossing parameter (siddon.cuh
// holds the same with an FP32 walk state).
__device__ __forceinline__ void ogs(bool dgs, double tmin, double t_min, double tmax, double t_max, unsigned &vmin,
                                    unsigned &vmax, double &t0, int &u, double diff, double b, double d, double s,
                                    unsigned n) {
    if (dgs) dgs_precomp(tmin, t_min, tmax, t_max, vmin, vmax, t0, u, diff, b, d, s, n);
    else sgd_precomp(tmin, t_min, tmax, t_max, vmin, vmax, t0, u, diff, b, d, s, n);
}

struct Walk {
    int ti, tj, tk, ux, uy, uz;
    double tx0, ty0, tz0, txu, tyu, tzu, tc;
    unsigned np;
    bool xy;
};

__device__ __forceinline__ bool pre2(double b1, double b2, double diff1, double diff2, double max1, double max2,
                                     double d1, double d2, int n1, int n2, int &t1, int &t2, double &t10, double &t20,
                                     double &t1u, double &t2u, int &u1, int &u2, unsigned &np, double xs, double ys,
                                     double xd, double yd, double &tc, bool &entry1) {
    const double apx = b1 - xs, apy = b2 - ys;
    t10 = apx / diff1;
    t20 = apy / diff2;
    const double txb = (max1 - xs) / diff1, tyb = (max2 - ys) / diff2;
    const double txmin = fmin(t10, txb), txmax = fmax(t10, txb), tymin = fmin(t20, tyb), tymax = fmax(t20, tyb);
    tc = fmax(txmin, tymin);
    const double tmax = fmin(txmax, tymax);
    entry1 = (tc == t10 || tc == txb);
    if (tc >= tmax) return true;
    unsigned imin, imax, jmin, jmax;
    ogs(xs < xd, tc, txmin, tmax, txmax, imin, imax, t10, u1, diff1, b1, d1, xs, (unsigned)n1);
    ogs(ys < yd, tc, tymin, tmax, tymax, jmin, jmax, t20, u2, diff2, b2, d2, ys, (unsigned)n2);
    np = imax + 1u + jmax + 1u - imin - jmin;
    const double pt = (fmin(t10, t20) + tc) / 2.0;
    t1 = (int)((pt * diff1 - apx) / d1);
    t2 = (int)((pt * diff2 - apy) / d2);
    t1u = d1 / fabs(diff1);
    t2u = d2 / fabs(diff2);
    return t1 < 0 || t2 < 0 || t1 >= n1 || t2 >= n2;
}

// The oblique-ray set-up (siddon_pre_loop_2D / 3D with their ORTH parts) in FP64.
__device__ __forceinline__ bool orth_setup(const Grid &g, const D3 &s, const D3 &d, const D3 &diff, Walk &w) {
    const double bx = g.bx, by = g.by, bz = g.bz, dx = g.dx, dy = g.dy, dz = g.dz;
    const double mx = bx + (double)g.nx * dx, my = by + (double)g.ny * dy, mz = bz + (double)g.nz * dz;
    w.ti = w.tj = w.tk = w.ux = w.uy = w.uz = 0;
    w.txu = w.tyu = w.tzu = w.tc = 0.0;
    w.tx0 = w.ty0 = w.tz0 = 1e8;
    w.np = 0u;
    w.xy = true;
    bool skip, e1;
    if (fabs(diff.z) < 1e-6) {
        w.tk = (int)(fabs(s.z - bz) / dz);
        if (w.tk < 0 || w.tk >= g.nz) return true;
        skip = pre2(bx, by, diff.x, diff.y, mx, my, dx, dy, g.nx, g.ny, w.ti, w.tj, w.tx0, w.ty0, w.txu, w.tyu, w.ux,
                    w.uy, w.np, s.x, s.y, d.x, d.y, w.tc, e1);
        w.xy = e1;
    } else if (fabs(diff.y) < 1e-6) {
        w.tj = perpendicular_start(by, d.y, dy, g.ny);
        skip = pre2(bx, bz, diff.x, diff.z, mx, mz, dx, dz, g.nx, g.nz, w.ti, w.tk, w.tx0, w.tz0, w.txu, w.tzu, w.ux,
                    w.uz, w.np, s.x, s.z, d.x, d.z, w.tc, e1);
        w.xy = true;
        if (d.y > my || d.y < by) skip = true;
    } else if (fabs(diff.x) < 1e-6) {
        w.ti = perpendicular_start(bx, d.x, dx, g.nx);
        skip = pre2(by, bz, diff.y, diff.z, my, mz, dy, dz, g.ny, g.nz, w.tj, w.tk, w.ty0, w.tz0, w.tyu, w.tzu, w.uy,
                    w.uz, w.np, s.y, s.z, d.y, d.z, w.tc, e1);
        w.xy = false;
        if (d.x > mx || d.x < bx) skip = true;
    } else {
        const D3 ap{bx - s.x, by - s.y, bz - s.z};
        D3 t0{ap.x / diff.x, ap.y / diff.y, ap.z / diff.z};
        const D3 tb{(mx - s.x) / diff.x, (my - s.y) / diff.y, (mz - s.z) / diff.z};
        const D3 mn{fmin(t0.x, tb.x), fmin(t0.y, tb.y), fmin(t0.z, tb.z)};
        const D3 mxv{fmax(t0.x, tb.x), fmax(t0.y, tb.y), fmax(t0.z, tb.z)};
        w.tc = fmax(fmax(mn.x, mn.z), mn.y);
        const double tmax = fmin(fmin(mxv.x, mxv.z), mxv.y);
        if (w.tc >= tmax) return true;
        unsigned imin, imax, jmin, jmax, kmin, kmax;
        ogs(s.x < d.x, w.tc, mn.x, tmax, mxv.x, imin, imax, t0.x, w.ux, diff.x, bx, dx, s.x, (unsigned)g.nx);
        ogs(s.y < d.y, w.tc, mn.y, tmax, mxv.y, jmin, jmax, t0.y, w.uy, diff.y, by, dy, s.y, (unsigned)g.ny);
        ogs(s.z < d.z, w.tc, mn.z, tmax, mxv.z, kmin, kmax, t0.z, w.uz, diff.z, bz, dz, s.z, (unsigned)g.nz);
        w.np = (kmax - kmin + 1u) + (jmax - jmin + 1u) + (imax - imin + 1u);
        const double pt = (fmin(fmin(t0.z, t0.y), t0.x) + w.tc) / 2.0;
        w.ti = (int)fmin(fmax((pt * diff.x - ap.x) / dx, 0.0), (double)(g.nx - 1));
        w.tj = (int)fmin(fmax((pt * diff.y - ap.y) / dy, 0.0), (double)(g.ny - 1));
        w.tk = (int)fmin(fmax((pt * diff.z - ap.z) / dz, 0.0), (double)(g.nz - 1));
        w.tx0 = t0.x; w.ty0 = t0.y; w.tz0 = t0.z;
        w.txu = dx / fabs(diff.x); w.tyu = dy / fabs(diff.y); w.tzu = dz / fabs(diff.z);
        // slices along x when the ray lies within 45 degrees of the x axis (the
        // reference's float thresholds, compared in FP64)
        const double ang = fabs(acos(diff.x / sqrt(diff.x * diff.x + diff.y * diff.y)));
        w.xy = (ang < (double)0.785398f && ang > 0.0) || (ang > (double)2.35619f && ang < (double)3.92699f) ||
               (ang > (double)5.497787f);
        skip = false;
    }
    return skip;
}

// Traces one PET ray through its tube: vis(linear_index, weight, tof_w, tof_sum)
// for every voxel inside.  `temp` gets the ray's scale (type 3: 1 / TotV)
// times the global factor.  Returns false when the ray is skipped.
template <int NB, class Visit>
__device__ bool orth_trace(const Grid &g, const Orth &o, const Ray &ray, float global_factor, const Tof &tof,
                           float &temp, Visit &&vis) {
    const D3 s{ray.s.x, ray.s.y, ray.s.z}, d{ray.d.x, ray.d.y, ray.d.z};
    const D3 diff{d.x - s.x, d.y - s.y, d.z - s.z};
    if ((diff.x == 0.0 && diff.y == 0.0) || isinf(diff.x) || isinf(diff.y) || isinf(diff.z) || isnan(diff.x) ||
        isnan(diff.y) || isnan(diff.z))
        return false;
    const double L = sqrt(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
    const double r2 = (double)o.width * (double)o.width;
    temp = (o.type == 3 ? (float)(1.0 / (L * (1.0 / 3.14159265358979323846) * r2)) : 1.f) * global_factor;
    float w[NB > 1 ? NB : 1];
    float tsum = 1.f;
    auto put = [&](int64_t ind, float ele) { vis(ind, ele, w, tsum); };
    OrthRay r;
    r.orl = o.type == 2 ? L * (double)o.width : L;
    r.cut2 = o.type == 3 ? (double)o.bmax * (double)o.bmax * r.orl * r.orl
                         : (1.0 - kThr) * (1.0 - kThr) * r.orl * r.orl;
    r.inv_orl = (float)(1.0 / r.orl);
    r.nxy = (int64_t)g.nx * g.ny;
    int tempk_b = 0;
    const double bx = g.bx, by = g.by, bz = g.bz, dxg = g.dx, dyg = g.dy, dzg = g.dz;
    const double mx = bx + (double)g.nx * dxg, my = by + (double)g.ny * dyg;

    if (fabs(diff.z) < 1e-6 && (fabs(diff.y) < 1e-6 || fabs(diff.x) < 1e-6)) {
        const int tk = (int)(fabs(s.z - bz) / dzg);
        if (tk < 0 || tk >= g.nz) return false;
        bool along_x;
        int nrow, row;
        double b1, d1;
        if (fabs(diff.y) < 1e-6 && d.y <= my && d.y >= by && s.y <= my && s.y >= by) {
            along_x = true;
            nrow = g.nx;
            b1 = bx; d1 = dxg;
            r.b1 = bx; r.d1 = dxg;
            r.b2 = by; r.d2 = dyg;
            r.sx = s.x; r.sy = s.y; r.sz = s.z;
            r.fx = diff.x; r.fy = diff.y; r.fz = diff.z;
            r.n1 = g.nx;
            r.st_slice = 1; r.st_in = g.nx;
            row = perpendicular_start(by, d.y, dyg, g.ny);
        } else if (fabs(diff.x) < 1e-6 && d.x <= mx && d.x >= bx && s.x <= mx && s.x >= bx) {
            along_x = false;
            nrow = g.ny;
            b1 = by; d1 = dyg;
            r.b1 = by; r.d1 = dyg;
            r.b2 = bx; r.d2 = dxg;
            r.sx = s.y; r.sy = s.x; r.sz = s.z;
            r.fx = diff.y; r.fy = diff.x; r.fz = diff.z;
            r.n1 = g.ny;
            r.st_slice = g.nx; r.st_in = 1;
            row = perpendicular_start(bx, d.x, dxg, g.nx);
        } else {
            return false;
        }
        // the voxels between the end points (projectorType123.cl:541-576)
        int x1 = 0, x2 = nrow - 1;
        double dT1 = d1, dT2 = d1;
        {
            const double sa = along_x ? s.x : s.y, da = along_x ? d.x : d.y;
            double dist1, dist2;
            if (sa > da) { dist1 = b1 - da; dist2 = b1 + (double)nrow * d1 - sa; }
            else { dist1 = b1 - sa; dist2 = b1 + (double)nrow * d1 - da; }
            if (dist1 < 0.0) {
                const int kk = (int)ceil(-dist1 / d1);
                if (kk < nrow) { x1 = kk; dT1 = fmin(dist1 + (double)kk * d1, d1); }
            }
            if (dist2 > 0.0) {
                const int mm = (int)ceil(dist2 / d1);
                const int kk = nrow - 1 - mm;
                if (kk >= x1) { x2 = kk; dT2 = fmin((double)mm * d1 - dist2, d1); }
            }
        }
        float D = 0.f, ddsign = 0.f;
        if (NB > 1) {
            D = (float)((d1 * (double)nrow) / copysign(2.0, along_x ? diff.y : diff.x));
            ddsign = sgnf(D);
        }
        for (int ii = x1; ii <= x2; ++ii) {
            if (NB > 1) {
                double d_in = d1;
                if (x1 > 0 && ii == x1) d_in = dT1;
                else if (x2 < nrow - 1 && ii == x2) d_in = dT2;
                tsum = tof_weights<NB>(tof, ddsign, (float)d_in, D, w);
            }
            orth_slice(o, g, r, ii, row, tk, false, tempk_b, 0, put);
            if (NB > 1) D -= (float)d1 * ddsign;
        }
        return true;
    }

    Walk wk;
    if (orth_setup(g, s, d, diff, wk)) return false;
    float D = 0.f, ddsign = 0.f;
    if (NB > 1) {
        const double a = diff.x * wk.tc, b = diff.y * wk.tc, c = diff.z * wk.tc;
        D = (float)(sqrt(a * a + b * b + c * c) - L / 2.0);
        ddsign = sgnf(D);
    }
    int nslice;
    if (!wk.xy) {
        int t;
        double tt;
        t = wk.ti; wk.ti = wk.tj; wk.tj = t;
        t = wk.ux; wk.ux = wk.uy; wk.uy = t;
        tt = wk.tx0; wk.tx0 = wk.ty0; wk.ty0 = tt;
        tt = wk.txu; wk.txu = wk.tyu; wk.tyu = tt;
        r.sx = s.y; r.sy = s.x; r.sz = s.z;
        r.fx = diff.y; r.fy = diff.x; r.fz = diff.z;
        r.b1 = by; r.d1 = dyg;
        r.b2 = bx; r.d2 = dxg;
        nslice = g.ny; r.n1 = g.nx;
        r.st_slice = g.nx; r.st_in = 1;
    } else {
        r.sx = s.x; r.sy = s.y; r.sz = s.z;
        r.fx = diff.x; r.fy = diff.y; r.fz = diff.z;
        r.b1 = bx; r.d1 = dxg;
        r.b2 = by; r.d2 = dyg;
        nslice = g.nx; r.n1 = g.ny;
        r.st_slice = 1; r.st_in = g.nx;
    }
    int ti_a = wk.ti, tj_a = wk.tj, tk_a = wk.tk, told = 0;
    double tc = wk.tc;
    for (unsigned ii = 0; ii < wk.np; ++ii) {
        ti_a = wk.ti; tj_a = wk.tj; tk_a = wk.tk;
        const double tx0_a = wk.tx0, ty0_a = wk.ty0, tz0_a = wk.tz0;
        double t0;
        if (wk.tz0 < wk.ty0 && wk.tz0 < wk.tx0) {
            t0 = wk.tz0; wk.tk += wk.uz; wk.tz0 += wk.tzu;
        } else if (wk.ty0 < wk.tx0) {
            t0 = wk.ty0; wk.tj += wk.uy; wk.ty0 += wk.tyu;
        } else {
            t0 = wk.tx0; wk.ti += wk.ux; wk.tx0 += wk.txu;
        }
        const bool pass = (t0 >= 0.0 && t0 <= 1.0) || (tc >= 0.0 && tc <= 1.0);
        const float ele = pass ? (float)((fmin(t0, 1.0) - fmax(tc, 0.0)) * L) : 0.f;
        tc = t0;
        if (NB > 1) tsum = tof_weights<NB>(tof, ddsign, ele, D, w);
        if (ii == 0) {
            tempk_b = tk_a;
            if (wk.ux >= 0) {
                for (int kk = ti_a - 1; kk >= 0; --kk)
                    if (orth_slice(o, g, r, kk, tj_a, tempk_b, true, tempk_b, wk.uz, put) == 0) break;
            } else {
                for (int kk = ti_a + 1; kk < nslice; ++kk)
                    if (orth_slice(o, g, r, kk, tj_a, tempk_b, true, tempk_b, wk.uz, put) == 0) break;
            }
        }
        if (tz0_a >= tx0_a && ty0_a >= tx0_a) {
            orth_slice(o, g, r, ti_a, tj_a, tk_a, false, tempk_b, wk.uz, put);
            told = ti_a;
        }
        if (NB > 1) D -= ele * ddsign;
        if (wk.ti < 0 || wk.ti >= nslice || wk.tj < 0 || wk.tj >= r.n1 || wk.tk < 0 || wk.tk >= g.nz) break;
    }
    if (wk.ux < 0) {
        if (told != ti_a) ti_a++;
        for (int kk = ti_a - 1; kk >= 0; --kk)
            if (orth_slice(o, g, r, kk, tj_a, tk_a, false, tempk_b, wk.uz, put) == 0) break;
    } else {
        if (told != ti_a) ti_a--;
        for (int kk = ti_a + 1; kk < nslice; ++kk)
            if (orth_slice(o, g, r, kk, tj_a, tk_a, false, tempk_b, wk.uz, put) == 0) break;
    }
    return true;
}

// Register caps: 64 per thread for the forward projection (8 CTAs, 32 warps per SM) and 80 for the
// backprojection (6 CTAs); the tracer is latency-bound on dependent FP64 arithmetic, and the extra warps
// hide more of it than the spills to the stack cost.
template <int NB>
__global__ void __launch_bounds__(kBlockO, 8) k_orth_fp(Grid g, RaySet rs, Orth o, Tof tof, float gf, const float *img,
                                                     float *y) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rs.m_size) return;
    const Ray ray = load_ray(rs, r);
    float ax[NB];
#pragma unroll
    for (int to = 0; to < NB; ++to) ax[to] = 0.f;
    float temp = 0.f;
    const bool ok = orth_trace<NB>(g, o, ray, gf, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
        const float v = ele * __ldg(img + ind);
        if (NB == 1) {
            ax[0] += v;
        } else {
#pragma unroll
            for (int to = 0; to < NB; ++to) ax[to] += w[to] * (v / tsum);
        }
    });
    const float corr = ok && (rs.w || rs.mu) ? ray_correction(g, rs, ray, r) : 1.f;
#pragma unroll
    for (int to = 0; to < NB; ++to) y[r + to * rs.m_size] = ok ? ax[to] * temp * corr : 0.f;
}

template <int NB>
__global__ void __launch_bounds__(kBlockO, 6) k_orth_bp(Grid g, RaySet rs, Orth o, Tof tof, float gf, const float *y,
                                                     float *img, float *sens) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rs.m_size) return;
    float yr[NB];
    bool any = sens != nullptr;
#pragma unroll
    for (int to = 0; to < NB; ++to) {
        yr[to] = y ? __ldg(y + r + to * rs.m_size) : 0.f;
        any |= yr[to] != 0.f;
    }
    if (!any) return;
    const Ray ray = load_ray(rs, r);
    const float corr = (rs.w || rs.mu) ? ray_correction(g, rs, ray, r) : 1.f;
    // the ray's scale is known before the trace: recompute it the way orth_trace does
    const double fx = (double)ray.d.x - ray.s.x, fy = (double)ray.d.y - ray.s.y, fz = (double)ray.d.z - ray.s.z;
    const double L = sqrt(fx * fx + fy * fy + fz * fz);
    const double r2 = (double)o.width * (double)o.width;
    const float scale = (o.type == 3 ? (float)(1.0 / (L * (1.0 / 3.14159265358979323846) * r2)) : 1.f) * gf * corr;
    float temp;
    orth_trace<NB>(g, o, ray, gf, tof, temp, [&](int64_t ind, float ele, const float *w, float tsum) {
        const float le = ele * scale;
        float yax, val;
        if (NB == 1) {
            yax = yr[0] * le;
            val = le;
        } else {
            const float dX = le / tsum;
            yax = 0.f;
            val = 0.f;
#pragma unroll
            for (int to = 0; to < NB; ++to) {
                const float a = dX * w[to];
                val += a;
                yax += a * yr[to];
            }
        }
        if (img) atomicAdd(img + ind, yax);
        if (sens) atomicAdd(sens + ind, val);
    });
}

// The non-TOF tube weights of each ray (the backprojection's ele x scale) for the transposed system matrix:
// the count of every voxel's entries, then the atomic fill (sysmat.cu sorts and slices the lists).
__device__ __forceinline__ float orth_ray_scale(const Orth &o, const RaySet &rs, const Grid &g, const Ray &ray,
                                                int64_t r, float gf) {
    const float corr = (rs.w || rs.mu) ? ray_correction(g, rs, ray, r) : 1.f;
    const double fx = (double)ray.d.x - ray.s.x, fy = (double)ray.d.y - ray.s.y, fz = (double)ray.d.z - ray.s.z;
    const double L = sqrt(fx * fx + fy * fy + fz * fz);
    const double r2 = (double)o.width * (double)o.width;
    return (o.type == 3 ? (float)(1.0 / (L * (1.0 / 3.14159265358979323846) * r2)) : 1.f) * gf * corr;
}

__global__ void __launch_bounds__(kBlockO, 6) k_orth_sm_count(Grid g, RaySet rs, Orth o, float gf,
                                                              unsigned *__restrict__ cnt, unsigned *__restrict__ rcnt) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rs.m_size) return;
    const Ray ray = load_ray(rs, r);
    const float scale = orth_ray_scale(o, rs, g, ray, r, gf);
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    float temp;
    unsigned k = 0;
    orth_trace<1>(g, o, ray, gf, tof, temp, [&](int64_t ind, float ele, const float *, float) {
        const float le = ele * scale;
        if (isnan(le) || le == 0.f) return;
        atomicAdd(cnt + ind, 1u);
        ++k;
    });
    rcnt[r] = k;
}

// rsent (or NULL): the ray-major copy in slices of 32 rays, entry k of ray l of slice s at rsoff[s] + 32 k + l
__global__ void __launch_bounds__(kBlockO, 6) k_orth_sm_fill(Grid g, RaySet rs, Orth o, float gf,
                                                             unsigned long long *__restrict__ cursor,
                                                             uint2 *__restrict__ ent, const int64_t *__restrict__ rsoff,
                                                             uint2 *__restrict__ rsent) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rs.m_size) return;
    const Ray ray = load_ray(rs, r);
    const float scale = orth_ray_scale(o, rs, g, ray, r, gf);
    const Tof tof{1, 0.f, 0.f, 0.f, nullptr};
    float temp;
    uint2 *rd = rsent ? rsent + rsoff[r >> 5] + (r & 31) : nullptr;
    int64_t k = 0;
    orth_trace<1>(g, o, ray, gf, tof, temp, [&](int64_t ind, float ele, const float *, float) {
        const float le = ele * scale;
        if (isnan(le) || le == 0.f) return;
        const unsigned long long pos = atomicAdd(cursor + ind, 1ull);
        ent[pos] = make_uint2((unsigned)r, __float_as_uint(le));
        if (rd) rd[32 * k] = make_uint2((unsigned)ind, __float_as_uint(le));
        ++k;
    });
}

template <int NB>
int launch_fp(const Grid &g, const RaySet &rs, const Orth &o, const Tof &tof, float gf, const float *img, float *y,
              cudaStream_t st) {
    const unsigned blocks = (unsigned)((rs.m_size + kBlockO - 1) / kBlockO);
    k_orth_fp<NB><<<blocks, kBlockO, 0, st>>>(g, rs, o, tof, gf, img, y);
    OMB_LAUNCH_CHECK("orthogonal / volume forward projection launch");
    return OMB_OK;
}

template <int NB>
int launch_bp(const Grid &g, const RaySet &rs, const Orth &o, const Tof &tof, float gf, const float *y, float *img,
              float *sens, cudaStream_t st) {
    const unsigned blocks = (unsigned)((rs.m_size + kBlockO - 1) / kBlockO);
    k_orth_bp<NB><<<blocks, kBlockO, 0, st>>>(g, rs, o, tof, gf, y, img, sens);
    OMB_LAUNCH_CHECK("orthogonal / volume backprojection launch");
    return OMB_OK;
}

}  // namespace

#define OMB_ORTH_NB(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

int orth_forward(const Grid &g, const RaySet &rs, const Orth &o, const Tof &tof, float gf, const float *img, float *y,
                 cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    switch (tof.nbins) {
#define OMB_CASE(N) \
    case N: return launch_fp<N>(g, rs, o, tof, gf, img, y, st);
        OMB_ORTH_NB(OMB_CASE)
#undef OMB_CASE
        default: return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
}

int orth_sm_count(const Grid &g, const RaySet &rs, const Orth &o, float gf, unsigned *cnt, unsigned *rcnt,
                  cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    k_orth_sm_count<<<(unsigned)((rs.m_size + kBlockO - 1) / kBlockO), kBlockO, 0, st>>>(g, rs, o, gf, cnt, rcnt);
    OMB_LAUNCH_CHECK("tube system matrix count launch");
    return OMB_OK;
}

int orth_sm_fill(const Grid &g, const RaySet &rs, const Orth &o, float gf, unsigned long long *cursor, uint2 *ent,
                 const int64_t *rsoff, uint2 *rsent, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    k_orth_sm_fill<<<(unsigned)((rs.m_size + kBlockO - 1) / kBlockO), kBlockO, 0, st>>>(g, rs, o, gf, cursor, ent,
                                                                                        rsoff, rsent);
    OMB_LAUNCH_CHECK("tube system matrix fill launch");
    return OMB_OK;
}

int orth_backward(const Grid &g, const RaySet &rs, const Orth &o, const Tof &tof, float gf, const float *y, float *img,
                  float *sens, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    switch (tof.nbins) {
#define OMB_CASE(N) \
    case N: return launch_bp<N>(g, rs, o, tof, gf, y, img, sens, st);
        OMB_ORTH_NB(OMB_CASE)
#undef OMB_CASE
        default: return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
}

}  // namespace omb
