// Improved Siddon ray traversal (projector type 1), device side.
//
// Restates the ray set-up and voxel walk of OMEGA's projectorType123.cl
// (-DSIDDON; lines 81-1374) with its helpers in general_opencl_functions.h:
// getDetectorCoordinatesFullSinogram (1601), getDetectorCoordinatesCT (1325),
// getIndex (914), perpendicular_start / perpendicular_elements (1673-1760),
// d_g_s_precomp / s_g_d_precomp (1763-1820), compute_element (1834),
// siddon_pre_loop_2D (1853) / _3D (1916), TOF weights (1077-1117),
// denominator (1155) and rhs (1212).
//
// Differences from the reference kernel, all deliberate:
//  * parametric positions along the ray are t0 + n*tu (one FMA from an
//    integer step count) instead of a running sum, so FP32 rounding does not
//    accumulate along long oblique rays;
//  * the per-ray set-up (entry/exit parameters, first voxel, intersection
//    count, in-plane row bounds) runs in FP64 -- rays entering exactly on a
//    voxel corner lose their first voxel, or the whole ray, to FP32 rounding
//    in the reference algorithm; the per-voxel walk stays FP32;
//  * divisions are IEEE (no --use_fast_math); TOF exponentials use __expf;
//  * the in-plane perpendicular backprojection addresses voxel (i, j, k) as
//    i + j*Nx + k*Nx*Ny for every image shape (the reference's linear index
//    there uses Ny as the row stride, which equals Nx only for square images);
//  * image reads are read-only-cache loads instead of a point-sampled 3-D
//    texture (identical values for the in-range indices the walk produces).
#pragma once

#include "common.cuh"

namespace omb {

__device__ __forceinline__ float sgnf(float v) { return (float)((0.f < v) - (v < 0.f)); }

struct Ray {
    float3 s, d;
};

// Ray end points of launch-local ray `r`; also returns the measurement index
// (output position) of the ray in the launch's output vector.
__device__ __forceinline__ Ray load_ray(const RaySet &rs, int64_t r) {
    Ray ray;
    if (rs.modality == OMB_PET_LISTMODE) {
        const float *q = rs.xy + (rs.proj0 + r) * 6;
        ray.s = make_float3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
        ray.d = make_float3(__ldg(q + 3), __ldg(q + 4), __ldg(q + 5));
        return ray;
    }
    if (rs.modality == OMB_PET_INDEXED) {
        const int64_t e = (rs.proj0 + r) * 2;
        const int t0 = __ldg(rs.tr + e), t1 = __ldg(rs.tr + e + 1);
        const int a0 = __ldg(rs.ax + e), a1 = __ldg(rs.ax + e + 1);
        ray.s = make_float3(__ldg(rs.xy + 2 * t0), __ldg(rs.xy + 2 * t0 + 1), __ldg(rs.z + a0));
        ray.d = make_float3(__ldg(rs.xy + 2 * t1), __ldg(rs.xy + 2 * t1 + 1), __ldg(rs.z + a1));
        return ray;
    }
    int64_t ix, iy, iz;
    if (rs.stype == 0) {
        const int64_t nbin = (int64_t)rs.n_rows * rs.n_cols;
        if (r <= 0x7fffffff && nbin <= 0x7fffffff) {
            // 32-bit division (the 64-bit one is a long software routine)
            const unsigned ru = (unsigned)r, nb = (unsigned)nbin;
            const unsigned z32 = ru / nb, b = ru - z32 * nb;
            const unsigned y32 = b / (unsigned)rs.n_rows;
            iz = z32;
            iy = y32;
            ix = b - y32 * (unsigned)rs.n_rows;
        } else {
            iz = r / nbin;
            const int64_t b = r - iz * nbin;
            iy = b / rs.n_rows;
            ix = b - iy * rs.n_rows;
        }
        iz += rs.proj0;
    } else {
        // Measurement-level subsets (general_opencl_functions.h:914-940):
        // the launch's k-th ray is sinogram element k*S + s of the chosen order.
        const int64_t S = rs.n_subsets, nr = rs.n_rows, nc = rs.n_cols;
        int64_t x = r;
        if (rs.stype == 1) {
            x = x * S + rs.cur_subset;
            iy = x % nc;
            iz = x / (nr * nc);
            ix = (x / nc) % nr;
        } else if (rs.stype == 2) {
            x = x * S + rs.cur_subset;
            iz = x / (nr * nc);
            iy = (x / nr) % nc;
            ix = x % nr;
        } else if (rs.stype == 4) {
            x = (x / nr) * nr * S + nr * rs.cur_subset + x % nr;
            iz = x / (nr * nc);
            iy = (x / nr) % nc;
            ix = x % nr;
        } else {  // 5
            iy = x % nc;
            x = x / nc * S + rs.cur_subset;
            iz = x / nr;
            ix = x % nr;
        }
    }
    if (rs.modality == OMB_PET_SINOGRAM) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(rs.xy) + (ix + iy * rs.n_rows));
        const float2 zz = __ldg(reinterpret_cast<const float2 *>(rs.z) + iz);
        ray.s = make_float3(q.x, q.y, zz.x);
        ray.d = make_float3(q.z, q.w, zz.y);
    } else {
        const float *p = rs.xy + iz * 6;
        ray.s = make_float3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
        float3 d = make_float3(__ldg(p + 3), __ldg(p + 4), __ldg(p + 5));
        const float ux = __ldg(rs.z + iz * 2), uy = __ldg(rs.z + iz * 2 + 1);
        const float ia = (float)ix - (float)rs.n_rows / 2.f + .5f;
        const float ib = (float)iy - (float)rs.n_cols / 2.f + .5f;
        d.x += ia * ux;
        d.y += ia * uy;
        d.z += ib * rs.pitch_y;
        ray.d = d;
    }
    return ray;
}

// Ray lorZ x lorXY of a multi-ray LOR (multirayCoordinateShiftZ / XY,
// general_opencl_functions.h:1120-1140): both end points moved by the same
// offset, the rays spaced evenly over the crystal, axial shift first.
__device__ __forceinline__ Ray multiray_shift(Ray ray, const RaySet &rs, int lor_xy, int lor_z) {
    if (rs.nr_z > 1) {
        float interval = rs.cr_z / (float)(rs.nr_z * 2);
        ray.s.z += (interval - rs.cr_z / 2.f);
        ray.d.z += (interval - rs.cr_z / 2.f);
        interval *= 2.f;
        ray.s.z += interval * lor_z;
        ray.d.z += interval * lor_z;
    }
    if (rs.nr_xy > 1) {
        float interval = rs.cr_xy / (float)(rs.nr_xy * 2);
        const float c = interval - rs.cr_xy / 2.f;
        ray.s.x += c;
        ray.d.x += c;
        ray.s.y += c;
        ray.d.y += c;
        interval *= 2.f;
        ray.s.x += interval * lor_xy;
        ray.d.x += interval * lor_xy;
        ray.s.y += interval * lor_xy;
        ray.d.y += interval * lor_xy;
    }
    return ray;
}

__device__ __forceinline__ int perpendicular_start(double b, double d, double dd, int n) {
    int t = (int)floor((d - b) / dd);
    if (t < 0 || t >= n) t = 0;
    return t;
}

// Entry voxel bounds along one axis when the source coordinate is below the
// detector's (Jacobs et al. eqs. 11-14) -- d_g_s_precomp.  FP64: these
// decide where a ray starts and how many voxels it crosses, and rays that
// enter exactly on a voxel corner (common for crystals on the grid axes)
// resolve differently in FP32.
__device__ __forceinline__ void dgs_precomp(double tmin, double t_min, double tmax, double t_max, unsigned &vmin,
                                            unsigned &vmax, double &t0, int &u, double diff, double b, double d,
                                            double s, unsigned n) {
    if (tmin == t_min) {
        vmin = 1u;
    } else {
        const double pt = s + tmin * diff;
        vmin = __double2uint_ru((pt - b) / d);
    }
    if (tmax == t_max) {
        vmax = n;
    } else {
        const double pt = s + tmax * diff;
        vmax = __double2uint_rd((pt - b) / d);
    }
    t0 += ((double)vmin * d) / diff;
    u = 1;
}

// Same when the source coordinate is above the detector's (eqs. 15-18) -- s_g_d_precomp.
__device__ __forceinline__ void sgd_precomp(double tmin, double t_min, double tmax, double t_max, unsigned &vmin,
                                            unsigned &vmax, double &t0, int &u, double diff, double b, double d,
                                            double s, unsigned n) {
    if (tmin == t_min) {
        vmax = n - 1u;
    } else {
        const double pt = s + tmin * diff;
        vmax = __double2uint_rd((pt - b) / d);
    }
    if (tmax == t_max) {
        vmin = 0u;
    } else {
        const double pt = s + tmax * diff;
        vmin = __double2uint_ru((pt - b) / d);
    }
    t0 += ((double)vmax * d) / diff;
    u = -1;
}

// Per-axis walk state: next boundary t0 + n*tu (FP32, from the FP64 set-up).
struct Axis {
    float t0;   // first boundary crossing
    float tu;   // spacing of boundary crossings
    int n;      // crossings taken
    int u;      // voxel step (+1/-1, 0 when the ray does not advance on this axis)
    __device__ __forceinline__ float next() const { return fmaf((float)n, tu, t0); }
};

// 2-D pre-loop (siddon_pre_loop_2D) in FP64: fills the two moving axes.
// Returns true when the ray misses the grid.
__device__ __forceinline__ bool pre_loop_2d(double b1, double b2, double diff1, double diff2, double max1,
                                            double max2, double d1, double d2, int n1, int n2, int &t1, int &t2,
                                            Axis &a1, Axis &a2, unsigned &np, double xs, double ys, double xd,
                                            double yd, double &tc) {
    const double apu_tx = b1 - xs;
    const double apu_ty = b2 - ys;
    double t10 = apu_tx / diff1;
    double t20 = apu_ty / diff2;
    const double txback = (max1 - xs) / diff1;
    const double tyback = (max2 - ys) / diff2;
    const double txmin = fmin(t10, txback), txmax = fmax(t10, txback);
    const double tymin = fmin(t20, tyback), tymax = fmax(t20, tyback);
    tc = fmax(txmin, tymin);
    const double tmax = fmin(txmax, tymax);
    if (tc >= tmax) return true;
    unsigned imin, imax, jmin, jmax;
    if (xs < xd)
        dgs_precomp(tc, txmin, tmax, txmax, imin, imax, t10, a1.u, diff1, b1, d1, xs, (unsigned)n1);
    else
        sgd_precomp(tc, txmin, tmax, txmax, imin, imax, t10, a1.u, diff1, b1, d1, xs, (unsigned)n1);
    if (ys < yd)
        dgs_precomp(tc, tymin, tmax, tymax, jmin, jmax, t20, a2.u, diff2, b2, d2, ys, (unsigned)n2);
    else
        sgd_precomp(tc, tymin, tmax, tymax, jmin, jmax, t20, a2.u, diff2, b2, d2, ys, (unsigned)n2);
    np = imax + 1u + jmax + 1u - imin - jmin;
    const double pt = (fmin(t10, t20) + tc) / 2.0;
    t1 = (int)((pt * diff1 - apu_tx) / d1);
    t2 = (int)((pt * diff2 - apu_ty) / d2);
    a1.t0 = (float)t10;
    a1.tu = (float)(d1 / fabs(diff1));
    a1.n = 0;
    a2.t0 = (float)t20;
    a2.tu = (float)(d2 / fabs(diff2));
    a2.n = 0;
    if (t1 < 0 || t2 < 0 || t1 >= n1 || t2 >= n2) return true;
    return false;
}

struct D3 {
    double x, y, z;
};

// 3-D pre-loop (siddon_pre_loop_3D) in FP64.
__device__ __forceinline__ bool pre_loop_3d(const Grid &g, D3 s, D3 d, D3 diff, int &ti, int &tj, int &tk, Axis &ax,
                                            Axis &ay, Axis &az, unsigned &np, double &tc) {
    const double mx = (double)g.mx, my = (double)g.my, mz = (double)g.mz;
    const double bx = (double)g.bx, by = (double)g.by, bz = (double)g.bz;
    const double dx = (double)g.dx, dy = (double)g.dy, dz = (double)g.dz;
    const D3 apuT{bx - s.x, by - s.y, bz - s.z};
    D3 t0{apuT.x / diff.x, apuT.y / diff.y, apuT.z / diff.z};
    const D3 tb{(mx - s.x) / diff.x, (my - s.y) / diff.y, (mz - s.z) / diff.z};
    const D3 tmn{fmin(t0.x, tb.x), fmin(t0.y, tb.y), fmin(t0.z, tb.z)};
    const D3 tmx{fmax(t0.x, tb.x), fmax(t0.y, tb.y), fmax(t0.z, tb.z)};
    tc = fmax(fmax(tmn.x, tmn.z), tmn.y);
    const double tmax = fmin(fmin(tmx.x, tmx.z), tmx.y);
    if (tc >= tmax) return true;
    unsigned imin, imax, jmin, jmax, kmin, kmax;
    if (s.x < d.x)
        dgs_precomp(tc, tmn.x, tmax, tmx.x, imin, imax, t0.x, ax.u, diff.x, bx, dx, s.x, (unsigned)g.nx);
    else
        sgd_precomp(tc, tmn.x, tmax, tmx.x, imin, imax, t0.x, ax.u, diff.x, bx, dx, s.x, (unsigned)g.nx);
    if (s.y < d.y)
        dgs_precomp(tc, tmn.y, tmax, tmx.y, jmin, jmax, t0.y, ay.u, diff.y, by, dy, s.y, (unsigned)g.ny);
    else
        sgd_precomp(tc, tmn.y, tmax, tmx.y, jmin, jmax, t0.y, ay.u, diff.y, by, dy, s.y, (unsigned)g.ny);
    if (s.z < d.z)
        dgs_precomp(tc, tmn.z, tmax, tmx.z, kmin, kmax, t0.z, az.u, diff.z, bz, dz, s.z, (unsigned)g.nz);
    else
        sgd_precomp(tc, tmn.z, tmax, tmx.z, kmin, kmax, t0.z, az.u, diff.z, bz, dz, s.z, (unsigned)g.nz);
    np = (kmax - kmin + 1u) + (jmax - jmin + 1u) + (imax - imin + 1u);
    const double pt = (fmin(fmin(t0.z, t0.y), t0.x) + tc) / 2.0;
    ti = (int)fmin(fmax((pt * diff.x - apuT.x) / dx, 0.0), (double)(g.nx - 1));
    tj = (int)fmin(fmax((pt * diff.y - apuT.y) / dy, 0.0), (double)(g.ny - 1));
    tk = (int)fmin(fmax((pt * diff.z - apuT.z) / dz, 0.0), (double)(g.nz - 1));
    ax.t0 = (float)t0.x; ax.tu = (float)(dx / fabs(diff.x)); ax.n = 0;
    ay.t0 = (float)t0.y; ay.tu = (float)(dy / fabs(diff.y)); ay.n = 0;
    az.t0 = (float)t0.z; az.tu = (float)(dz / fabs(diff.z)); az.n = 0;
    return false;
}

// TOF weights of one element (TOFLoop/TOFWeight/normPDF): 4-point trapezoid
// of the Gaussian over the element, per bin centre.  Returns the sum clamped
// to >= epps.
template <int NB>
__device__ __forceinline__ float tof_weights(const Tof &tof, float ddsign, float element, float D, float *w) {
    const float dX = element / 3.f;  // TRAPZ_BINS - 1
    // the trapezoid points in units of sigma sqrt(2): a_tr = (D - c) / (sigma sqrt 2) - tr * beta (the last one
    // at the element's end), each Gaussian exp(-a^2); the normalisation sigma_coef * dX applied once to the
    // weighted sum of the four
    const float si = tof.sigma_inv * 0.70710678f;
    const float beta = dX * ddsign * si;
    const float aend = element * ddsign * si;
    const float scale = tof.sigma_coef * dX;
    float sum = 0.f;
#pragma unroll
    for (int to = 0; to < NB; ++to) {
        const float a0 = (D - __ldg(tof.centers + to)) * si;
        const float a1 = a0 - beta, a2 = fmaf(-2.f, beta, a0), a3 = a0 - aend;
        const float e0 = __expf(-(a0 * a0)), e1 = __expf(-(a1 * a1));
        const float e2 = __expf(-(a2 * a2)), e3 = __expf(-(a3 * a3));
        w[to] = ((e0 + e3) + 2.f * (e1 + e2)) * scale;
        sum += w[to];
    }
    if (sum < tof.epps) sum = tof.epps;
    return sum;
}

// Walks one ray through the grid and calls vis(linear_voxel_index, length,
// tof_weights, tof_sum) for every intersected voxel.  `temp` receives the
// ray's normalisation (1/L * global_factor for PET, 1 for CT).  Returns false
// when the ray contributes nothing.
//
// K > 1 (non-TOF only) takes the crossings K at a time: the K voxel indices
// and lengths are computed first and the K visits follow in straight-line
// code, so a gathering visitor has K independent loads in flight instead of
// waiting on one per voxel.  Steps past the ray's end are visited with length
// 0 at the batch's first (valid) voxel.  The visits and their order are those
// of K = 1.
//
// FULL_ROW: a ray along an image row visits every voxel of the row at full
// voxel length (the row attenuation sum of the reference's CPU projector,
// projector_functions.h:1193-1205) instead of the part between its end points.
template <int NB, int K = 1, bool FULL_ROW = false, class Visit>
__device__ __forceinline__ bool siddon_walk(const Grid &g, const Ray &ray, bool pet, float global_factor,
                                            const Tof &tof, float &temp, Visit &&vis) {
    // Set-up in FP64 (end points are FP32, so their differences are exact);
    // the per-voxel walk below runs in FP32.
    const D3 s{ray.s.x, ray.s.y, ray.s.z}, d{ray.d.x, ray.d.y, ray.d.z};
    const D3 diff{d.x - s.x, d.y - s.y, d.z - s.z};
    if ((diff.x == 0.0 && diff.y == 0.0) || isinf(diff.x) || isinf(diff.y) || isinf(diff.z) || isnan(diff.x) ||
        isnan(diff.y) || isnan(diff.z))
        return false;
    const double Ld = sqrt(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
    const float L = (float)Ld;
    temp = pet ? (float)(1.0 / Ld) * global_factor : 1.f;
    const int64_t nxy = (int64_t)g.nx * g.ny;
    float w[NB > 1 ? NB : 1];
    const double bx = g.bx, by = g.by, bz = g.bz, dxg = g.dx, dyg = g.dy, dzg = g.dz;
    const double mx = g.mx, my = g.my, mz = g.mz;

    if (fabs(diff.z) < 1e-6 && (fabs(diff.y) < 1e-6 || fabs(diff.x) < 1e-6)) {
        // In-plane ray parallel to a grid axis: every voxel of one row.
        const int tk = (int)(fabs(s.z - bz) / dzg);
        if (tk < 0 || tk >= g.nz) return false;
        int x1, x2, nrow, n0;
        double dT1, dT2, d_b, dd, d_db, d_d2;
        bool along_x;
        if (fabs(diff.y) < 1e-6 && d.y <= my && d.y >= by && s.y <= my && s.y >= by) {
            along_x = true;
            nrow = g.nx;
            x1 = 0; x2 = g.nx - 1; dT1 = dxg; dT2 = dxg;
            double dist1, dist2;
            if (s.x > d.x) { dist1 = bx - d.x; dist2 = bx + (double)g.nx * dxg - s.x; }
            else           { dist1 = bx - s.x; dist2 = bx + (double)g.nx * dxg - d.x; }
            if (dist1 < 0.0) {
                const int kk = (int)ceil(-dist1 / dxg);
                if (kk < g.nx) { x1 = kk; dT1 = fmin(dist1 + (double)kk * dxg, dxg); }
            }
            if (dist2 > 0.0) {
                const int mm = (int)ceil(dist2 / dxg);
                const int kk = g.nx - 1 - mm;
                if (kk >= x1) { x2 = kk; dT2 = fmin((double)mm * dxg - dist2, dxg); }
            }
            d_b = by; dd = d.y; d_db = dyg; d_d2 = dxg; n0 = g.ny;
        } else if (fabs(diff.x) < 1e-6 && d.x <= mx && d.x >= bx && s.x <= mx && s.x >= bx) {
            along_x = false;
            nrow = g.ny;
            x1 = 0; x2 = g.ny - 1; dT1 = dyg; dT2 = dyg;
            double dist1, dist2;
            if (s.y > d.y) { dist1 = by - d.y; dist2 = by + (double)g.ny * dyg - s.y; }
            else           { dist1 = by - s.y; dist2 = by + (double)g.ny * dyg - d.y; }
            if (dist1 < 0.0) {
                const int kk = (int)ceil(-dist1 / dyg);
                if (kk < g.ny) { x1 = kk; dT1 = fmin(dist1 + (double)kk * dyg, dyg); }
            }
            if (dist2 > 0.0) {
                const int mm = (int)ceil(dist2 / dyg);
                const int kk = g.ny - 1 - mm;
                if (kk >= x1) { x2 = kk; dT2 = fmin((double)mm * dyg - dist2, dyg); }
            }
            d_b = bx; dd = d.x; d_db = dxg; d_d2 = dyg; n0 = g.nx;
        } else {
            return false;
        }
        const int row = perpendicular_start(d_b, dd, d_db, n0);
        // voxel (i, j, k): along x -> (ii, row, tk); along y -> (row, ii, tk)
        const int64_t base = (int64_t)tk * nxy + (along_x ? (int64_t)row * g.nx : (int64_t)row);
        const int64_t stride = along_x ? 1 : g.nx;
        const float fd2 = (float)d_d2, fT1 = (float)dT1, fT2 = (float)dT2;
        // TOF along a row: the reference CPU projector's form
        // (projector_functions.h:1617-1685): D starts at +-half the row length
        // with the sign of the near-zero transverse component taken by
        // copysign (the GPU kernel's sign(diff.y) is 0 for rows parallel to x
        // and would put the ray in the centre bin), and the normalisation
        // integrates a full voxel width.
        float D = 0.f, ddsign = 0.f;
        if (NB > 1) {
            D = (float)((d_d2 * (double)nrow) / copysign(2.0, along_x ? diff.y : diff.x));
            ddsign = sgnf(D);
        }
        // FULL_ROW: from voxel 0 to the row's end
        for (int ii = FULL_ROW ? 0 : x1; ii <= (FULL_ROW ? nrow - 1 : x2); ++ii) {
            if (FULL_ROW) {
                vis(base + (int64_t)ii * stride, fd2, w, 1.f);
                continue;
            }
            float d_in = fd2;
            if (x1 > 0 && ii == x1) d_in = fT1;
            else if (x2 < nrow - 1 && ii == x2) d_in = fT2;
            float tsum = 1.f;
            if (NB > 1) {
                tsum = tof_weights<NB>(tof, ddsign, fd2, D, w);
                if (d_in != fd2) tof_weights<NB>(tof, ddsign, d_in, D, w);
            }
            vis(base + (int64_t)ii * stride, d_in, w, tsum);
            if (NB > 1) D -= fd2 * ddsign;
        }
        return true;
    }

    int ti = 0, tj = 0, tk = 0;
    Axis ax{1e8f, 0.f, 0, 0}, ay{1e8f, 0.f, 0, 0}, az{1e8f, 0.f, 0, 0};
    unsigned np = 0u;
    double tcd = 0.0;
    bool skip;
    if (fabs(diff.z) < 1e-6) {
        tk = (int)(fabs(s.z - bz) / dzg);
        if (tk < 0 || tk >= g.nz) return false;
        skip = pre_loop_2d(bx, by, diff.x, diff.y, mx, my, dxg, dyg, g.nx, g.ny, ti, tj, ax, ay, np, s.x, s.y, d.x,
                           d.y, tcd);
    } else if (fabs(diff.y) < 1e-6) {
        tj = perpendicular_start(by, d.y, dyg, g.ny);
        skip = pre_loop_2d(bx, bz, diff.x, diff.z, mx, mz, dxg, dzg, g.nx, g.nz, ti, tk, ax, az, np, s.x, s.z, d.x,
                           d.z, tcd);
        if (d.y > my || d.y < by) skip = true;
    } else if (fabs(diff.x) < 1e-6) {
        ti = perpendicular_start(bx, d.x, dxg, g.nx);
        skip = pre_loop_2d(by, bz, diff.y, diff.z, my, mz, dyg, dzg, g.ny, g.nz, tj, tk, ay, az, np, s.y, s.z, d.y,
                           d.z, tcd);
        if (d.x > mx || d.x < bx) skip = true;
    } else {
        skip = pre_loop_3d(g, s, d, diff, ti, tj, tk, ax, ay, az, np, tcd);
    }
    if (skip) return false;

    float D = 0.f, ddsign = 0.f;
    if (NB > 1) {
        const double a = diff.x * tcd, b = diff.y * tcd, c = diff.z * tcd;
        D = (float)(sqrt(a * a + b * b + c * c) - Ld / 2.0);
        ddsign = sgnf(D);
    }
    float tc = (float)tcd;
    float tx = ax.next(), ty = ay.next(), tz = az.next();
    if constexpr (K > 1) {
        static_assert(NB == 1, "batched crossings are built for non-TOF walks");
        bool done = false;
        for (unsigned ii = 0u; ii < np && !done; ii += K) {
            int64_t inds[K];
            float eles[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                inds[k] = k ? inds[0] : 0;
                eles[k] = 0.f;
                if (!done && ii + k < np) {
                    inds[k] = (int64_t)tj * g.nx + ti + (int64_t)tk * nxy;
                    float t0;
                    if (tz < ty && tz < tx) {
                        t0 = tz;
                        tk += az.u;
                        az.n++;
                        tz = az.next();
                    } else if (ty < tx) {
                        t0 = ty;
                        tj += ay.u;
                        ay.n++;
                        ty = ay.next();
                    } else {
                        t0 = tx;
                        ti += ax.u;
                        ax.n++;
                        tx = ax.next();
                    }
                    const bool pass = (t0 >= 0.f && t0 <= 1.f) || (tc >= 0.f && tc <= 1.f);
                    eles[k] = pass ? (fminf(t0, 1.f) - fmaxf(tc, 0.f)) * L : 0.f;
                    tc = t0;
                    done = ti < 0 || ti >= g.nx || tj < 0 || tj >= g.ny || tk < 0 || tk >= g.nz;
                }
            }
#pragma unroll
            for (int k = 0; k < K; ++k) vis(inds[k], eles[k], w, 1.f);
        }
    } else {
        for (unsigned ii = 0u; ii < np; ++ii) {
            const int64_t ind = (int64_t)tj * g.nx + ti + (int64_t)tk * nxy;
            float t0;
            if (tz < ty && tz < tx) {
                t0 = tz;
                tk += az.u;
                az.n++;
                tz = az.next();
            } else if (ty < tx) {
                t0 = ty;
                tj += ay.u;
                ay.n++;
                ty = ay.next();
            } else {
                t0 = tx;
                ti += ax.u;
                ax.n++;
                tx = ax.next();
            }
            const bool pass = (t0 >= 0.f && t0 <= 1.f) || (tc >= 0.f && tc <= 1.f);
            const float ele = pass ? (fminf(t0, 1.f) - fmaxf(tc, 0.f)) * L : 0.f;
            tc = t0;
            float tsum = 1.f;
            if (NB > 1) tsum = tof_weights<NB>(tof, ddsign, ele, D, w);
            vis(ind, ele, w, tsum);
            if (NB > 1) D -= ele * ddsign;
            if (ti < 0 || ti >= g.nx || tj < 0 || tj >= g.ny || tk < 0 || tk >= g.nz) break;
        }
    }
    return true;
}

// Per-ray correction factor of PET rays (projector_functions.h:1754-1832):
// the measurement's multiplicative weight (normalisation x scatter x LOR
// attenuation, premultiplied by the caller) and, with an attenuation image,
// exp(-sum of mu x intersection length) along the ray.  1 without either.
__device__ __forceinline__ float ray_correction(const Grid &g, const RaySet &rs, const Ray &ray, int64_t r) {
    float f = rs.w ? __ldg(rs.w + r) : 1.f;
    if (rs.mu) {
        const Tof tof1{1, 0.f, 0.f, 0.f, nullptr};
        float jel = 0.f, t;
        siddon_walk<1, 1, true>(g, ray, true, 1.f, tof1, t, [&](int64_t ind, float ele, const float *, float) {
            jel += ele * -__ldg(rs.mu + ind);
        });
        f *= expf(jel);
    }
    return f;
}

}  // namespace omb
