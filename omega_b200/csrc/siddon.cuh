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
    int64_t ix, iy, iz;
    if (rs.stype == 0) {
        const int64_t nbin = (int64_t)rs.n_rows * rs.n_cols;
        iz = r / nbin;
        const int64_t b = r - iz * nbin;
        iy = b / rs.n_rows;
        ix = b - iy * rs.n_rows;
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
    Ray ray;
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

__device__ __forceinline__ int perpendicular_start(float b, float d, float dd, int n) {
    int t = (int)floorf((d - b) / dd);
    if (t < 0 || t >= n) t = 0;
    return t;
}

// Entry voxel bounds along one axis when the source coordinate is below the
// detector's (Jacobs et al. eqs. 11-14) -- d_g_s_precomp.
__device__ __forceinline__ void dgs_precomp(float tmin, float t_min, float tmax, float t_max, unsigned &vmin,
                                            unsigned &vmax, float &t0, int &u, float diff, float b, float d,
                                            float s, unsigned n) {
    if (tmin == t_min) {
        vmin = 1u;
    } else {
        const float pt = s + tmin * diff;
        vmin = __float2uint_ru((pt - b) / d);
    }
    if (tmax == t_max) {
        vmax = n;
    } else {
        const float pt = s + tmax * diff;
        vmax = __float2uint_rd((pt - b) / d);
    }
    t0 += ((float)vmin * d) / diff;
    u = 1;
}

// Same when the source coordinate is above the detector's (eqs. 15-18) -- s_g_d_precomp.
__device__ __forceinline__ void sgd_precomp(float tmin, float t_min, float tmax, float t_max, unsigned &vmin,
                                            unsigned &vmax, float &t0, int &u, float diff, float b, float d,
                                            float s, unsigned n) {
    if (tmin == t_min) {
        vmax = n - 1u;
    } else {
        const float pt = s + tmin * diff;
        vmax = __float2uint_rd((pt - b) / d);
    }
    if (tmax == t_max) {
        vmin = 0u;
    } else {
        const float pt = s + tmax * diff;
        vmin = __float2uint_ru((pt - b) / d);
    }
    t0 += ((float)vmax * d) / diff;
    u = -1;
}

// Per-axis walk state: next boundary t0 + n*tu.
struct Axis {
    float t0;   // first boundary crossing
    float tu;   // spacing of boundary crossings
    int n;      // crossings taken
    int u;      // voxel step (+1/-1, 0 when the ray does not advance on this axis)
    __device__ __forceinline__ float next() const { return fmaf((float)n, tu, t0); }
};

// 2-D pre-loop (siddon_pre_loop_2D): fills the two moving axes.  Returns true
// when the ray misses the grid.
__device__ __forceinline__ bool pre_loop_2d(float b1, float b2, float diff1, float diff2, float max1, float max2,
                                            float d1, float d2, int n1, int n2, int &t1, int &t2, Axis &a1,
                                            Axis &a2, unsigned &np, float xs, float ys, float xd, float yd,
                                            float &tc) {
    const float apu_tx = b1 - xs;
    const float apu_ty = b2 - ys;
    float t10 = apu_tx / diff1;
    float t20 = apu_ty / diff2;
    const float txback = (max1 - xs) / diff1;
    const float tyback = (max2 - ys) / diff2;
    const float txmin = fminf(t10, txback), txmax = fmaxf(t10, txback);
    const float tymin = fminf(t20, tyback), tymax = fmaxf(t20, tyback);
    tc = fmaxf(txmin, tymin);
    const float tmax = fminf(txmax, tymax);
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
    const float pt = (fminf(t10, t20) + tc) / 2.f;
    t1 = __float2int_rz((pt * diff1 - apu_tx) / d1);
    t2 = __float2int_rz((pt * diff2 - apu_ty) / d2);
    a1.t0 = t10;
    a1.tu = d1 / fabsf(diff1);
    a1.n = 0;
    a2.t0 = t20;
    a2.tu = d2 / fabsf(diff2);
    a2.n = 0;
    if (t1 < 0 || t2 < 0 || t1 >= n1 || t2 >= n2) return true;
    return false;
}

// 3-D pre-loop (siddon_pre_loop_3D).
__device__ __forceinline__ bool pre_loop_3d(const Grid &g, float3 s, float3 d, float3 diff, int &ti, int &tj,
                                            int &tk, Axis &ax, Axis &ay, Axis &az, unsigned &np, float &tc) {
    const float3 apuT = make_float3(g.bx - s.x, g.by - s.y, g.bz - s.z);
    float3 t0 = make_float3(apuT.x / diff.x, apuT.y / diff.y, apuT.z / diff.z);
    const float3 tb = make_float3((g.mx - s.x) / diff.x, (g.my - s.y) / diff.y, (g.mz - s.z) / diff.z);
    const float3 tmn = make_float3(fminf(t0.x, tb.x), fminf(t0.y, tb.y), fminf(t0.z, tb.z));
    const float3 tmx = make_float3(fmaxf(t0.x, tb.x), fmaxf(t0.y, tb.y), fmaxf(t0.z, tb.z));
    tc = fmaxf(fmaxf(tmn.x, tmn.z), tmn.y);
    const float tmax = fminf(fminf(tmx.x, tmx.z), tmx.y);
    if (tc >= tmax) return true;
    unsigned imin, imax, jmin, jmax, kmin, kmax;
    if (s.x < d.x)
        dgs_precomp(tc, tmn.x, tmax, tmx.x, imin, imax, t0.x, ax.u, diff.x, g.bx, g.dx, s.x, (unsigned)g.nx);
    else
        sgd_precomp(tc, tmn.x, tmax, tmx.x, imin, imax, t0.x, ax.u, diff.x, g.bx, g.dx, s.x, (unsigned)g.nx);
    if (s.y < d.y)
        dgs_precomp(tc, tmn.y, tmax, tmx.y, jmin, jmax, t0.y, ay.u, diff.y, g.by, g.dy, s.y, (unsigned)g.ny);
    else
        sgd_precomp(tc, tmn.y, tmax, tmx.y, jmin, jmax, t0.y, ay.u, diff.y, g.by, g.dy, s.y, (unsigned)g.ny);
    if (s.z < d.z)
        dgs_precomp(tc, tmn.z, tmax, tmx.z, kmin, kmax, t0.z, az.u, diff.z, g.bz, g.dz, s.z, (unsigned)g.nz);
    else
        sgd_precomp(tc, tmn.z, tmax, tmx.z, kmin, kmax, t0.z, az.u, diff.z, g.bz, g.dz, s.z, (unsigned)g.nz);
    np = (kmax - kmin + 1u) + (jmax - jmin + 1u) + (imax - imin + 1u);
    const float pt = (fminf(fminf(t0.z, t0.y), t0.x) + tc) / 2.f;
    const float fi = fminf(fmaxf(fmaf(pt, diff.x, -apuT.x) / g.dx, 0.f), (float)(g.nx - 1));
    const float fj = fminf(fmaxf(fmaf(pt, diff.y, -apuT.y) / g.dy, 0.f), (float)(g.ny - 1));
    const float fk = fminf(fmaxf(fmaf(pt, diff.z, -apuT.z) / g.dz, 0.f), (float)(g.nz - 1));
    ti = __float2int_rz(fi);
    tj = __float2int_rz(fj);
    tk = __float2int_rz(fk);
    ax.t0 = t0.x; ax.tu = g.dx / fabsf(diff.x); ax.n = 0;
    ay.t0 = t0.y; ay.tu = g.dy / fabsf(diff.y); ay.n = 0;
    az.t0 = t0.z; az.tu = g.dz / fabsf(diff.z); az.n = 0;
    return false;
}

// TOF weights of one element (TOFLoop/TOFWeight/normPDF): 4-point trapezoid
// of the Gaussian over the element, per bin centre.  Returns the sum clamped
// to >= epps.
template <int NB>
__device__ __forceinline__ float tof_weights(const Tof &tof, float ddsign, float element, float D, float *w) {
    const float dX = element / 3.f;  // TRAPZ_BINS - 1
    const float sdX = dX * ddsign;
    float sum = 0.f;
#pragma unroll
    for (int to = 0; to < NB; ++to) {
        const float c = __ldg(tof.centers + to);
        float a = (D - c) * tof.sigma_inv;
        float out = tof.sigma_coef * __expf(-0.5f * a * a);
#pragma unroll
        for (int tr = 1; tr < 3; ++tr) {
            a = (fmaf(-sdX, (float)tr, D) - c) * tof.sigma_inv;
            out += tof.sigma_coef * __expf(-0.5f * a * a) * 2.f;
        }
        a = (fmaf(-element, ddsign, D) - c) * tof.sigma_inv;
        out += tof.sigma_coef * __expf(-0.5f * a * a);
        w[to] = out * dX;
        sum += w[to];
    }
    if (sum < tof.epps) sum = tof.epps;
    return sum;
}

// Walks one ray through the grid and calls vis(linear_voxel_index, length,
// tof_weights, tof_sum) for every intersected voxel.  `temp` receives the
// ray's normalisation (1/L * global_factor for PET, 1 for CT).  Returns false
// when the ray contributes nothing.
template <int NB, class Visit>
__device__ __forceinline__ bool siddon_walk(const Grid &g, const Ray &ray, bool pet, float global_factor,
                                            const Tof &tof, float &temp, Visit &&vis) {
    const float3 s = ray.s, d = ray.d;
    const float3 diff = make_float3(d.x - s.x, d.y - s.y, d.z - s.z);
    if ((diff.x == 0.f && diff.y == 0.f) || isinf(diff.x) || isinf(diff.y) || isinf(diff.z) || isnan(diff.x) ||
        isnan(diff.y) || isnan(diff.z))
        return false;
    const float L = sqrtf(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
    temp = pet ? (1.f / L) * global_factor : 1.f;
    const int64_t nxy = (int64_t)g.nx * g.ny;
    float w[NB > 1 ? NB : 1];

    if (fabsf(diff.z) < 1e-6f && (fabsf(diff.y) < 1e-6f || fabsf(diff.x) < 1e-6f)) {
        // In-plane ray parallel to a grid axis: every voxel of one row.
        const int tk = (int)(fabsf(s.z - g.bz) / g.dz);
        if (tk < 0 || tk >= g.nz) return false;
        int x1, x2, nrow;
        float dT1, dT2, d_b, dd, d_db, d_d2;
        int n0;
        bool along_x;
        if (fabsf(diff.y) < 1e-6f && d.y <= g.my && d.y >= g.by && s.y <= g.my && s.y >= g.by) {
            along_x = true;
            nrow = g.nx;
            x1 = 0; x2 = g.nx - 1; dT1 = g.dx; dT2 = g.dx;
            float dist1, dist2;
            if (s.x > d.x) { dist1 = g.bx - d.x; dist2 = g.bx + (float)g.nx * g.dx - s.x; }
            else           { dist1 = g.bx - s.x; dist2 = g.bx + (float)g.nx * g.dx - d.x; }
            if (dist1 < 0.f) {
                const int kk = (int)ceilf(-dist1 / g.dx);
                if (kk < g.nx) { x1 = kk; dT1 = fminf(dist1 + (float)kk * g.dx, g.dx); }
            }
            if (dist2 > 0.f) {
                const int mm = (int)ceilf(dist2 / g.dx);
                const int kk = g.nx - 1 - mm;
                if (kk >= x1) { x2 = kk; dT2 = fminf((float)mm * g.dx - dist2, g.dx); }
            }
            d_b = g.by; dd = d.y; d_db = g.dy; d_d2 = g.dx; n0 = g.ny;
        } else if (fabsf(diff.x) < 1e-6f && d.x <= g.mx && d.x >= g.bx && s.x <= g.mx && s.x >= g.bx) {
            along_x = false;
            nrow = g.ny;
            x1 = 0; x2 = g.ny - 1; dT1 = g.dy; dT2 = g.dy;
            float dist1, dist2;
            if (s.y > d.y) { dist1 = g.by - d.y; dist2 = g.by + (float)g.ny * g.dy - s.y; }
            else           { dist1 = g.by - s.y; dist2 = g.by + (float)g.ny * g.dy - d.y; }
            if (dist1 < 0.f) {
                const int kk = (int)ceilf(-dist1 / g.dy);
                if (kk < g.ny) { x1 = kk; dT1 = fminf(dist1 + (float)kk * g.dy, g.dy); }
            }
            if (dist2 > 0.f) {
                const int mm = (int)ceilf(dist2 / g.dy);
                const int kk = g.ny - 1 - mm;
                if (kk >= x1) { x2 = kk; dT2 = fminf((float)mm * g.dy - dist2, g.dy); }
            }
            d_b = g.bx; dd = d.x; d_db = g.dx; d_d2 = g.dy; n0 = g.nx;
        } else {
            return false;
        }
        const int row = perpendicular_start(d_b, dd, d_db, n0);
        // voxel (i, j, k): along x -> (ii, row, tk); along y -> (row, ii, tk)
        const int64_t base = (int64_t)tk * nxy + (along_x ? (int64_t)row * g.nx : (int64_t)row);
        const int64_t stride = along_x ? 1 : g.nx;
        // TOF along a row: the reference CPU projector's form
        // (projector_functions.h:1617-1685): D starts at +-half the row length
        // with the sign of the near-zero transverse component taken by
        // copysign (the GPU kernel's sign(diff.y) is 0 for rows parallel to x
        // and would put the ray in the centre bin), and the normalisation
        // integrates a full voxel width.
        float D = 0.f, ddsign = 0.f;
        if (NB > 1) {
            D = (d_d2 * (float)nrow) / copysignf(2.f, along_x ? diff.y : diff.x);
            ddsign = sgnf(D);
        }
        for (int ii = x1; ii <= x2; ++ii) {
            float d_in = d_d2;
            if (x1 > 0 && ii == x1) d_in = dT1;
            else if (x2 < nrow - 1 && ii == x2) d_in = dT2;
            float tsum = 1.f;
            if (NB > 1) {
                tsum = tof_weights<NB>(tof, ddsign, d_d2, D, w);
                if (d_in != d_d2) tof_weights<NB>(tof, ddsign, d_in, D, w);
            }
            vis(base + (int64_t)ii * stride, d_in, w, tsum);
            if (NB > 1) D -= d_d2 * ddsign;
        }
        return true;
    }

    int ti = 0, tj = 0, tk = 0;
    Axis ax{1e8f, 0.f, 0, 0}, ay{1e8f, 0.f, 0, 0}, az{1e8f, 0.f, 0, 0};
    unsigned np = 0u;
    float tc = 0.f;
    bool skip;
    if (fabsf(diff.z) < 1e-6f) {
        tk = (int)(fabsf(s.z - g.bz) / g.dz);
        if (tk < 0 || tk >= g.nz) return false;
        skip = pre_loop_2d(g.bx, g.by, diff.x, diff.y, g.mx, g.my, g.dx, g.dy, g.nx, g.ny, ti, tj, ax, ay, np, s.x,
                           s.y, d.x, d.y, tc);
    } else if (fabsf(diff.y) < 1e-6f) {
        tj = perpendicular_start(g.by, d.y, g.dy, g.ny);
        skip = pre_loop_2d(g.bx, g.bz, diff.x, diff.z, g.mx, g.mz, g.dx, g.dz, g.nx, g.nz, ti, tk, ax, az, np, s.x,
                           s.z, d.x, d.z, tc);
        if (d.y > g.my || d.y < g.by) skip = true;
    } else if (fabsf(diff.x) < 1e-6f) {
        ti = perpendicular_start(g.bx, d.x, g.dx, g.nx);
        skip = pre_loop_2d(g.by, g.bz, diff.y, diff.z, g.my, g.mz, g.dy, g.dz, g.ny, g.nz, tj, tk, ay, az, np, s.y,
                           s.z, d.y, d.z, tc);
        if (d.x > g.mx || d.x < g.bx) skip = true;
    } else {
        skip = pre_loop_3d(g, s, d, diff, ti, tj, tk, ax, ay, az, np, tc);
    }
    if (skip) return false;

    float D = 0.f, ddsign = 0.f;
    if (NB > 1) {
        const float dxc = diff.x * tc, dyc = diff.y * tc, dzc = diff.z * tc;
        D = sqrtf(dxc * dxc + dyc * dyc + dzc * dzc) - L / 2.f;
        ddsign = sgnf(D);
    }
    float tx = ax.next(), ty = ay.next(), tz = az.next();
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
    return true;
}

}  // namespace omb
