/*
 * TEST INFRASTRUCTURE ONLY -- the FP64 checker for projector type 1.
 * Nothing in the product links or calls this file; tests/, the smoke check
 * and bench.py's CPU baseline load it as the oracle.
 *
 * CPU restatement, in double precision, of OMEGA's GPU improved-Siddon
 * projector (source/opencl/projectorType123.cl:81-1374 built with -DSIDDON,
 * -DTOTLENGTH, USEIMAGES point sampling) and the helpers it uses in
 * source/opencl/general_opencl_functions.h:
 *   getIndex 914-940, TOFDis/TOFWeight/TOFLoop/normPDF 1077-1117,
 *   denominator 1155-1185, rhs 1212-1275, getDetectorCoordinatesCT 1325-1410,
 *   getDetectorCoordinatesFullSinogram 1601-1628, perpendicular_start 1673,
 *   perpendicular_elements 1681-1760, d_g_s_precomp 1763, s_g_d_precomp 1793,
 *   compute_element 1834, siddon_pre_loop_2D 1853, siddon_pre_loop_3D 1916,
 *   forwardProjectAF 1961.
 * The in-plane perpendicular branch follows projectorType123.cl:514-780,
 * except its TOF set-up, which follows the reference CPU projector
 * (projector_functions.h:1617-1685) because the GPU kernel's sign(diff.y) is
 * zero for rows parallel to x.
 * Every ray is walked exactly as the kernel walks it (same branch order, same
 * thresholds, same running-sum parametric stepping) but in FP64, so it is the
 * reference answer the FP32 GPU kernels are measured against.
 * Built by oracle/Makefile into oracle/liboracle.so.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle_common.h"

static unsigned to_u_ceil(double v) {
    v = ceil(v);
    if (!(v > 0.0)) return 0u;
    if (v >= 4294967295.0) return 4294967295u;
    return (unsigned)v;
}

static unsigned to_u_floor(double v) {
    v = floor(v);
    if (!(v > 0.0)) return 0u;
    if (v >= 4294967295.0) return 4294967295u;
    return (unsigned)v;
}

static int perp_start(double b, double d, double dd, int n) {
    int t = (int)floor((d - b) / dd);
    if (t < 0 || t >= n) t = 0;
    return t;
}


static void dgs(double tmin, double t_min, double tmax, double t_max, unsigned *vmin, unsigned *vmax, double *t0,
                int *u, double diff, double b, double d, double s, unsigned n) {
    if (tmin == t_min) *vmin = 1u;
    else *vmin = to_u_ceil(((s + tmin * diff) - b) / d);
    if (tmax == t_max) *vmax = n;
    else *vmax = to_u_floor(((s + tmax * diff) - b) / d);
    *t0 += ((double)*vmin * d) / diff;
    *u = 1;
}

static void sgd(double tmin, double t_min, double tmax, double t_max, unsigned *vmin, unsigned *vmax, double *t0,
                int *u, double diff, double b, double d, double s, unsigned n) {
    if (tmin == t_min) *vmax = n - 1u;
    else *vmax = to_u_floor(((s + tmin * diff) - b) / d);
    if (tmax == t_max) *vmin = 0u;
    else *vmin = to_u_ceil(((s + tmax * diff) - b) / d);
    *t0 += ((double)*vmax * d) / diff;
    *u = -1;
}

static int pre2d_xy(double b1, double b2, double diff1, double diff2, double max1, double max2, double d1,
                    double d2, int n1, int n2, int *t1, int *t2, double *t1u, double *t2u, unsigned *np, double xs,
                    double ys, double xd, double yd, double *tc, int *u1, int *u2, double *t10, double *t20,
                    int *entry1) {
    double apx = b1 - xs, apy = b2 - ys;
    *t10 = apx / diff1;
    *t20 = apy / diff2;
    double txb = (max1 - xs) / diff1, tyb = (max2 - ys) / diff2;
    double txmin = fmin(*t10, txb), txmax = fmax(*t10, txb), tymin = fmin(*t20, tyb), tymax = fmax(*t20, tyb);
    *tc = fmax(txmin, tymin);
    double tmax = fmin(txmax, tymax);
    /* the ray enters through a face of the first axis (siddon_pre_loop_2D, ORTH) */
    if (entry1) *entry1 = (*tc == *t10 || *tc == txb);
    if (*tc >= tmax) return 1;
    unsigned imin, imax, jmin, jmax;
    if (xs < xd) dgs(*tc, txmin, tmax, txmax, &imin, &imax, t10, u1, diff1, b1, d1, xs, (unsigned)n1);
    else sgd(*tc, txmin, tmax, txmax, &imin, &imax, t10, u1, diff1, b1, d1, xs, (unsigned)n1);
    if (ys < yd) dgs(*tc, tymin, tmax, tymax, &jmin, &jmax, t20, u2, diff2, b2, d2, ys, (unsigned)n2);
    else sgd(*tc, tymin, tmax, tymax, &jmin, &jmax, t20, u2, diff2, b2, d2, ys, (unsigned)n2);
    *np = imax + 1u + jmax + 1u - imin - jmin;
    double pt = (fmin(*t10, *t20) + *tc) / 2.0;
    *t1 = (int)((pt * diff1 - apx) / d1);
    *t2 = (int)((pt * diff2 - apy) / d2);
    *t1u = d1 / fabs(diff1);
    *t2u = d2 / fabs(diff2);
    if (*t1 < 0 || *t2 < 0 || *t1 >= n1 || *t2 >= n2) return 1;
    return 0;
}

static int pre2d(double b1, double b2, double diff1, double diff2, double max1, double max2, double d1, double d2,
                 int n1, int n2, int *t1, int *t2, double *t1u, double *t2u, unsigned *np, double xs, double ys,
                 double xd, double yd, double *tc, int *u1, int *u2, double *t10, double *t20) {
    return pre2d_xy(b1, b2, diff1, diff2, max1, max2, d1, d2, n1, n2, t1, t2, t1u, t2u, np, xs, ys, xd, yd, tc, u1,
                    u2, t10, t20, NULL);
}

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int pre3d(const oracle_geom *g, double mx, double my, double mz, v3 s, v3 d, v3 diff, int *ti, int *tj,
                 int *tk, double *txu, double *tyu, double *tzu, unsigned *np, double *tc, int *ux, int *uy, int *uz,
                 double *tx0, double *ty0, double *tz0) {
    v3 ap = {g->bx - s.x, g->by - s.y, g->bz - s.z};
    v3 t0 = {ap.x / diff.x, ap.y / diff.y, ap.z / diff.z};
    v3 tb = {(mx - s.x) / diff.x, (my - s.y) / diff.y, (mz - s.z) / diff.z};
    v3 mn = {fmin(t0.x, tb.x), fmin(t0.y, tb.y), fmin(t0.z, tb.z)};
    v3 mxv = {fmax(t0.x, tb.x), fmax(t0.y, tb.y), fmax(t0.z, tb.z)};
    *tc = fmax(fmax(mn.x, mn.z), mn.y);
    double tmax = fmin(fmin(mxv.x, mxv.z), mxv.y);
    *tx0 = t0.x; *ty0 = t0.y; *tz0 = t0.z;
    if (*tc >= tmax) return 1;
    unsigned imin, imax, jmin, jmax, kmin, kmax;
    if (s.x < d.x) dgs(*tc, mn.x, tmax, mxv.x, &imin, &imax, tx0, ux, diff.x, g->bx, g->dx, s.x, (unsigned)g->nx);
    else sgd(*tc, mn.x, tmax, mxv.x, &imin, &imax, tx0, ux, diff.x, g->bx, g->dx, s.x, (unsigned)g->nx);
    if (s.y < d.y) dgs(*tc, mn.y, tmax, mxv.y, &jmin, &jmax, ty0, uy, diff.y, g->by, g->dy, s.y, (unsigned)g->ny);
    else sgd(*tc, mn.y, tmax, mxv.y, &jmin, &jmax, ty0, uy, diff.y, g->by, g->dy, s.y, (unsigned)g->ny);
    if (s.z < d.z) dgs(*tc, mn.z, tmax, mxv.z, &kmin, &kmax, tz0, uz, diff.z, g->bz, g->dz, s.z, (unsigned)g->nz);
    else sgd(*tc, mn.z, tmax, mxv.z, &kmin, &kmax, tz0, uz, diff.z, g->bz, g->dz, s.z, (unsigned)g->nz);
    *np = (kmax - kmin + 1u) + (jmax - jmin + 1u) + (imax - imin + 1u);
    double pt = (fmin(fmin(*tz0, *ty0), *tx0) + *tc) / 2.0;
    *ti = (int)clampd((pt * diff.x - ap.x) / g->dx, 0.0, (double)(g->nx - 1));
    *tj = (int)clampd((pt * diff.y - ap.y) / g->dy, 0.0, (double)(g->ny - 1));
    *tk = (int)clampd((pt * diff.z - ap.z) / g->dz, 0.0, (double)(g->nz - 1));
    *txu = g->dx / fabs(diff.x);
    *tyu = g->dy / fabs(diff.y);
    *tzu = g->dz / fabs(diff.z);
    return 0;
}


/* Visitor: called per intersected voxel with the element length and the TOF weights. */
typedef void (*visit_fn)(void *ctx, int64_t ind, double ele, const double *w, double tsum);

/* Walks ray r; returns 0 when the ray is skipped.  *temp gets the ray
 * normalisation.  full_row: a ray along an image row visits every voxel of
 * the row at full length (the reference CPU projector's row attenuation sum,
 * projector_functions.h:1193-1205). */
static int walk_ex(const oracle_geom *g, int64_t r, int lxy, int lz, double *temp, visit_fn vis, void *ctx,
                   int full_row) {
    v3 s, d;
    load_ray(g, r, &s, &d);
    multiray_shift(g, lxy, lz, &s, &d);
    const double mx = g->bx + (double)g->nx * g->dx;
    const double my = g->by + (double)g->ny * g->dy;
    const double mz = g->bz + (double)g->nz * g->dz;
    v3 diff = {d.x - s.x, d.y - s.y, d.z - s.z};
    if ((diff.x == 0.0 && diff.y == 0.0) || isinf(diff.x) || isinf(diff.y) || isinf(diff.z) || isnan(diff.x) ||
        isnan(diff.y) || isnan(diff.z))
        return 0;
    const double L = sqrt(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
    const int nrays = (g->nr_xy > 1 ? g->nr_xy : 1) * (g->nr_z > 1 ? g->nr_z : 1);
    *temp = g->modality != 1 ? (1.0 / (L * nrays)) * g->global_factor : 1.0;
    const int64_t nxy = (int64_t)g->nx * g->ny;
    double w[MAXB];
    const int tofon = g->nbins > 1;

    if (fabs(diff.z) < 1e-6 && (fabs(diff.y) < 1e-6 || fabs(diff.x) < 1e-6)) {
        int tk = (int)(fabs(s.z - g->bz) / g->dz);
        if (tk < 0 || tk >= g->nz) return 0;
        int x1, x2, nrow, n0, along_x;
        double dT1, dT2, d_b, dd, d_db, d_d2;
        if (fabs(diff.y) < 1e-6 && d.y <= my && d.y >= g->by && s.y <= my && s.y >= g->by) {
            along_x = 1; nrow = g->nx; x1 = 0; x2 = g->nx - 1; dT1 = g->dx; dT2 = g->dx;
            double dist1, dist2;
            if (s.x > d.x) { dist1 = g->bx - d.x; dist2 = g->bx + (double)g->nx * g->dx - s.x; }
            else { dist1 = g->bx - s.x; dist2 = g->bx + (double)g->nx * g->dx - d.x; }
            if (dist1 < 0.0) { int kk = (int)ceil(-dist1 / g->dx); if (kk < g->nx) { x1 = kk; dT1 = fmin(dist1 + kk * g->dx, g->dx); } }
            if (dist2 > 0.0) { int mm = (int)ceil(dist2 / g->dx); int kk = g->nx - 1 - mm; if (kk >= x1) { x2 = kk; dT2 = fmin(mm * g->dx - dist2, g->dx); } }
            d_b = g->by; dd = d.y; d_db = g->dy; d_d2 = g->dx; n0 = g->ny;
        } else if (fabs(diff.x) < 1e-6 && d.x <= mx && d.x >= g->bx && s.x <= mx && s.x >= g->bx) {
            along_x = 0; nrow = g->ny; x1 = 0; x2 = g->ny - 1; dT1 = g->dy; dT2 = g->dy;
            double dist1, dist2;
            if (s.y > d.y) { dist1 = g->by - d.y; dist2 = g->by + (double)g->ny * g->dy - s.y; }
            else { dist1 = g->by - s.y; dist2 = g->by + (double)g->ny * g->dy - d.y; }
            if (dist1 < 0.0) { int kk = (int)ceil(-dist1 / g->dy); if (kk < g->ny) { x1 = kk; dT1 = fmin(dist1 + kk * g->dy, g->dy); } }
            if (dist2 > 0.0) { int mm = (int)ceil(dist2 / g->dy); int kk = g->ny - 1 - mm; if (kk >= x1) { x2 = kk; dT2 = fmin(mm * g->dy - dist2, g->dy); } }
            d_b = g->bx; dd = d.x; d_db = g->dx; d_d2 = g->dy; n0 = g->nx;
        } else {
            return 0;
        }
        int row = perp_start(d_b, dd, d_db, n0);
        int64_t base = (int64_t)tk * nxy + (along_x ? (int64_t)row * g->nx : (int64_t)row);
        int64_t stride = along_x ? 1 : g->nx;
        double D = 0.0, ddsign = 0.0;
        /* TOF along a row follows the reference CPU projector
         * (projector_functions.h:1641-1685): copysign for the starting side,
         * normalisation over a full voxel width, weights over the element. */
        if (tofon) { D = (d_d2 * (double)nrow) / copysign(2.0, along_x ? diff.y : diff.x); ddsign = sgn(D); }
        if (full_row) {
            for (int ii = 0; ii < nrow; ++ii) vis(ctx, base + (int64_t)ii * stride, d_d2, w, 1.0);
            return 1;
        }
        for (int ii = x1; ii <= x2; ++ii) {
            double d_in = d_d2;
            if (x1 > 0 && ii == x1) d_in = dT1;
            else if (x2 < nrow - 1 && ii == x2) d_in = dT2;
            double tsum = 1.0;
            if (tofon) {
                tsum = tof_weights(g, ddsign, d_d2, D, w);
                if (d_in != d_d2) tof_weights(g, ddsign, d_in, D, w);
            }
            vis(ctx, base + (int64_t)ii * stride, d_in, w, tsum);
            if (tofon) D -= d_d2 * ddsign;
        }
        return 1;
    }

    int ti = 0, tj = 0, tk = 0, ux = 0, uy = 0, uz = 0;
    double txu = 0, tyu = 0, tzu = 0, tc = 0, tx0 = 1e8, ty0 = 1e8, tz0 = 1e8;
    unsigned np = 0;
    int skip;
    if (fabs(diff.z) < 1e-6) {
        tk = (int)(fabs(s.z - g->bz) / g->dz);
        if (tk < 0 || tk >= g->nz) return 0;
        skip = pre2d(g->bx, g->by, diff.x, diff.y, mx, my, g->dx, g->dy, g->nx, g->ny, &ti, &tj, &txu, &tyu, &np,
                     s.x, s.y, d.x, d.y, &tc, &ux, &uy, &tx0, &ty0);
    } else if (fabs(diff.y) < 1e-6) {
        tj = perp_start(g->by, d.y, g->dy, g->ny);
        skip = pre2d(g->bx, g->bz, diff.x, diff.z, mx, mz, g->dx, g->dz, g->nx, g->nz, &ti, &tk, &txu, &tzu, &np,
                     s.x, s.z, d.x, d.z, &tc, &ux, &uz, &tx0, &tz0);
        if (d.y > my || d.y < g->by) skip = 1;
    } else if (fabs(diff.x) < 1e-6) {
        ti = perp_start(g->bx, d.x, g->dx, g->nx);
        skip = pre2d(g->by, g->bz, diff.y, diff.z, my, mz, g->dy, g->dz, g->ny, g->nz, &tj, &tk, &tyu, &tzu, &np,
                     s.y, s.z, d.y, d.z, &tc, &uy, &uz, &ty0, &tz0);
        if (d.x > mx || d.x < g->bx) skip = 1;
    } else {
        skip = pre3d(g, mx, my, mz, s, d, diff, &ti, &tj, &tk, &txu, &tyu, &tzu, &np, &tc, &ux, &uy, &uz, &tx0, &ty0,
                     &tz0);
    }
    if (skip) return 0;
    double D = 0.0, ddsign = 0.0;
    if (tofon) {
        double a = diff.x * tc, b = diff.y * tc, c = diff.z * tc;
        D = sqrt(a * a + b * b + c * c) - L / 2.0;
        ddsign = sgn(D);
    }
    for (unsigned ii = 0; ii < np; ++ii) {
        int64_t ind = (int64_t)tj * g->nx + ti + (int64_t)tk * nxy;
        double *t0;
        double tu;
        int *tijk, u;
        if (tz0 < ty0 && tz0 < tx0) { t0 = &tz0; tu = tzu; tijk = &tk; u = uz; }
        else if (ty0 < tx0) { t0 = &ty0; tu = tyu; tijk = &tj; u = uy; }
        else { t0 = &tx0; tu = txu; tijk = &ti; u = ux; }
        int pass = (*t0 >= 0.0 && *t0 <= 1.0) || (tc >= 0.0 && tc <= 1.0);
        double ele = pass ? (fmin(*t0, 1.0) - fmax(tc, 0.0)) * L : 0.0;
        *tijk += u;
        tc = *t0;
        *t0 += tu;
        double tsum = 1.0;
        if (tofon) tsum = tof_weights(g, ddsign, ele, D, w);
        vis(ctx, ind, ele, w, tsum);
        if (tofon) D -= ele * ddsign;
        if (ti < 0 || ti >= g->nx || tj < 0 || tj >= g->ny || tk < 0 || tk >= g->nz) break;
    }
    return 1;
}

static int walk(const oracle_geom *g, int64_t r, double *temp, visit_fn vis, void *ctx) {
    return walk_ex(g, r, 0, 0, temp, vis, ctx, 0);
}

static int nr(int n) { return n > 1 ? n : 1; }

typedef struct { const double *mu; double jel; } atn_ctx;

static void atn_visit(void *c, int64_t ind, double ele, const double *w, double tsum) {
    (void)w; (void)tsum;
    atn_ctx *a = (atn_ctx *)c;
    a->jel += ele * -a->mu[ind];
}

/* Correction factor of PET ray r: its weight times exp(-line integral of mu). */
static double ray_corr(const oracle_geom *g, int64_t r, int lxy, int lz) {
    if (g->modality == 1) return 1.0;
    double f = g->w ? g->w[r] : 1.0;
    if (g->mu) {
        atn_ctx a = {g->mu, 0.0};
        double t;
        walk_ex(g, r, lxy, lz, &t, atn_visit, &a, 1);
        f *= exp(a.jel);
    }
    return f;
}

typedef struct { const double *img; double ax[MAXB]; int nb; } fp_ctx;

static void fp_visit(void *c, int64_t ind, double ele, const double *w, double tsum) {
    fp_ctx *f = (fp_ctx *)c;
    double v = ele * f->img[ind];
    if (f->nb == 1) f->ax[0] += v;
    else for (int to = 0; to < f->nb; ++to) f->ax[to] += w[to] * (v / tsum);
}

/* y[r + to*m_size] = (A img)[r, to] for the rays of the launch. */
int oracle_siddon_fp(const oracle_geom *g, const double *img, double *y) {
    if (g->nbins < 1 || g->nbins > MAXB) return -1;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < g->m_size; ++r) {
        double out[MAXB];
        for (int to = 0; to < g->nbins; ++to) out[to] = 0.0;
        for (int lz = 0; lz < nr(g->nr_z); ++lz)
            for (int lxy = 0; lxy < nr(g->nr_xy); ++lxy) {
                fp_ctx f;
                f.img = img;
                f.nb = g->nbins;
                for (int to = 0; to < g->nbins; ++to) f.ax[to] = 0.0;
                double temp = 0.0;
                int ok = walk_ex(g, r, lxy, lz, &temp, fp_visit, &f, 0);
                const double corr = ok ? ray_corr(g, r, lxy, lz) : 0.0;
                for (int to = 0; to < g->nbins; ++to) out[to] += ok ? f.ax[to] * temp * corr : 0.0;
            }
        for (int to = 0; to < g->nbins; ++to) y[r + to * g->m_size] = out[to];
    }
    return 0;
}

typedef struct { double *img, *sens; double ax[MAXB]; int nb; double temp; } bp_ctx;

static void bp_visit(void *c, int64_t ind, double ele, const double *w, double tsum) {
    bp_ctx *b = (bp_ctx *)c;
    double le = ele * b->temp, yax = 0.0, val = 0.0;
    if (b->nb == 1) {
        yax = b->ax[0] * le;
        val = le;
    } else {
        double dX = le / tsum;
        for (int to = 0; to < b->nb; ++to) {
            double a = dX * w[to];
            val += a;
            yax += a * b->ax[to];
        }
    }
    if (b->img) b->img[ind] += yax;
    if (b->sens) b->sens[ind] += val;
}

/* img += A^T y; sens += A^T 1 when sens is not NULL.  Serial (deterministic). */
int oracle_siddon_bp(const oracle_geom *g, const double *y, double *img, double *sens) {
    if (g->nbins < 1 || g->nbins > MAXB) return -1;
    for (int64_t r = 0; r < g->m_size; ++r) {
        bp_ctx b;
        b.img = img;
        b.sens = sens;
        b.nb = g->nbins;
        int any = sens != NULL;
        for (int to = 0; to < g->nbins; ++to) {
            b.ax[to] = y ? y[r + to * g->m_size] : 0.0;
            any |= b.ax[to] != 0.0;
        }
        if (!any) continue;
        const int nrays = nr(g->nr_xy) * nr(g->nr_z);
        for (int lz = 0; lz < nr(g->nr_z); ++lz)
            for (int lxy = 0; lxy < nr(g->nr_xy); ++lxy) {
                /* the visitor needs the ray's normalisation before the walk sets it */
                double temp = 0.0;
                v3 s, d;
                load_ray(g, r, &s, &d);
                multiray_shift(g, lxy, lz, &s, &d);
                double dxl = d.x - s.x, dyl = d.y - s.y, dzl = d.z - s.z;
                double L = sqrt(dxl * dxl + dyl * dyl + dzl * dzl);
                b.temp = g->modality != 1 ? (1.0 / (L * nrays)) * g->global_factor * ray_corr(g, r, lxy, lz) : 1.0;
                walk_ex(g, r, lxy, lz, &temp, bp_visit, &b, 0);
            }
    }
    return 0;
}

/* Voxel-intersection count Np of every ray (the walk length), for the
 * algorithmic-byte model of the roofline. */
static void count_visit(void *c, int64_t ind, double ele, const double *w, double tsum) {
    (void)ind; (void)ele; (void)w; (void)tsum;
    ++*(int64_t *)c;
}

int64_t oracle_siddon_count(const oracle_geom *g) {
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int64_t r = 0; r < g->m_size; ++r) {
        int64_t n = 0;
        double temp;
        walk(g, r, &temp, count_visit, &n);
        total += n;
    }
    return total;
}

/* ------------------------------------------------------------------------
 * Projector types 2 (orthogonal distance) and 3 (volume of intersection):
 * the tube-of-response tracer of projectorType123.cl built with -DORTH
 * (-DVOL for type 3) and -DCRYSTXY / -DCRYSTZ, PET: ray set-up 493-508
 * (orth_ray_length, TotV), in-plane rows 514-760, oblique rays 791-1296,
 * with orthDistance3D / orthogonalHelper3D / compute_element_orth_3D of
 * opencl_functions_orth3D.h:24-417 and the ORTH parts of
 * siddon_pre_loop_2D / 3D (general_opencl_functions.h:1853-1958).
 * Each slice the ray leaves through its slice face (x, or y when the ray is
 * closer to the y axis) is scanned outward from the ray's voxel, row by row
 * in z and both ways in the slice, until the normalised distance drops out
 * of the tube; the slices before the ray's first and after its last voxel
 * are scanned until one contributes nothing.
 *
 * cpu_mode restates the reference CPU projector instead
 * (projector_functions.h:972-1160, 1500-2028): its descending in-slice loop
 * evaluates the ascending loop's last index, which has just failed, so it
 * ends at its first step; its scans start at the unclamped row / column
 * (voxel centres outside the grid count as failing); TotV = L pi r^2; and
 * its post-loop TOF weights use the last step's element at the decremented
 * TOF distance.  That variant is what the compiled reference computes, so it
 * pins everything the two share.
 * ------------------------------------------------------------------------ */

#define ORTH_THR 0.01
#define ORTH_CC 1e3
#define ORTH_PI 3.14159265358979323846

typedef struct {
    const oracle_geom *g;
    v3 s, diff;                 /* slice axis first (swapped when the slices run along y) */
    double orl;                 /* orth_ray_length */
    double b2, d2;              /* in-slice axis */
    int n1;                     /* in-slice count (maksimiXY) */
    int64_t st_slice, st_in;    /* linear-index strides of the slice and in-slice axes */
    visit_fn vis;
    void *ctx;
    const double *w;
    double tsum;
} orth_t;

static int imaxi(int a, int b) { return a > b ? a : b; }
static int imini(int a, int b) { return a < b ? a : b; }

/* orthogonalHelper3D: 1 = outside the tube (stop), 0 = visited */
static int orth_voxel(orth_t *o, int slice, int uu, int zz, double lx, double ly, double lz) {
    const oracle_geom *g = o->g;
    if (g->cpu_mode && (uu < 0 || uu >= o->n1 || zz < 0 || zz >= g->nz)) return 1;
    const double cy = o->b2 + (double)uu * o->d2 + o->d2 / 2.0;
    const double x0 = cy - o->s.y;
    const double y1 = o->diff.z * x0 - ly;
    const double z1 = -o->diff.x * x0 + lz;
    const double n2 = lx * lx + y1 * y1 + z1 * z1;
    double ele;
    if (g->proj_type == 3) {
        double dd;
        if (g->cpu_mode) {
            dd = sqrt(n2) / o->orl;
            if (dd >= g->bmax) return 1;
        } else {
            if (n2 > g->bmax * g->bmax * o->orl * o->orl) return 1;
            dd = sqrt(n2) / o->orl;
        }
        if (dd < g->bmin) {
            ele = g->vmax;
        } else {
            double q = (dd - g->bmin) * ORTH_CC;
            int iv = (int)(g->cpu_mode ? round(q) : rint(q));
            if (iv > g->nv - 1) iv = g->nv - 1;   /* the table's last entry (the reference reads past it) */
            ele = g->V[iv];
        }
    } else {
        if (g->cpu_mode) {
            ele = 1.0 - sqrt(n2) / o->orl;
            if (ele <= ORTH_THR) return 1;
        } else {
            if (n2 >= (1.0 - ORTH_THR) * (1.0 - ORTH_THR) * o->orl * o->orl) return 1;
            ele = 1.0 - sqrt(n2) / o->orl;
        }
    }
    const int64_t ind = (int64_t)slice * o->st_slice + (int64_t)uu * o->st_in + (int64_t)zz * g->nx * g->ny;
    o->vis(o->ctx, ind, ele, o->w, o->tsum);
    return 0;
}

/* One z row of a slice: the in-slice scans.  Updates uu1 / uu2 / brk / count. */
static void orth_row(orth_t *o, int slice, int temp2, int zz, double apu1, double lz, int *uu1, int *uu2, int *brk,
                     int *count) {
    const oracle_geom *g = o->g;
    const double cz = g->bz + (double)zz * g->dz + g->dz / 2.0;
    const double z0 = cz - o->s.z;
    const double lx = o->diff.x * z0 - apu1;
    const double ly = o->diff.y * z0;
    if (!g->crystxy) {
        *uu1 = temp2;
        *brk = orth_voxel(o, slice, temp2, zz, lx, ly, lz);
        *uu2 = temp2 - 1;
        return;
    }
    for (*uu1 = g->cpu_mode ? temp2 : imaxi(temp2, 0); *uu1 < o->n1; ++*uu1) {
        *brk = orth_voxel(o, slice, *uu1, zz, lx, ly, lz);
        if (*brk) break;
        ++*count;
    }
    if (g->cpu_mode) {
        *uu2 = temp2 - 1;
        if (*uu2 >= 0) *brk = 1;
        return;
    }
    for (*uu2 = imini(temp2, o->n1) - 1; *uu2 >= 0; --*uu2) {
        *brk = orth_voxel(o, slice, *uu2, zz, lx, ly, lz);
        if (*brk) break;
        ++*count;
    }
}

/* orthDistance3D: returns the number of voxels visited in the slice. */
static int orth_slice(orth_t *o, int slice, double cx, int temp2, int tempk, int pre_step, int *k, int ku) {
    const oracle_geom *g = o->g;
    int count = 0, brk = 0, uu1 = 0, uu2 = 0, zz;
    const double v0 = cx - o->s.x;
    const double lz = o->diff.y * v0;
    const double apu1 = o->diff.z * v0;
    if (!g->crystz) {
        orth_row(o, slice, temp2, tempk, apu1, lz, &uu1, &uu2, &brk, &count);
        return count;
    }
    for (zz = g->cpu_mode ? tempk : imaxi(tempk, 0); zz < g->nz; ++zz) {
        orth_row(o, slice, temp2, zz, apu1, lz, &uu1, &uu2, &brk, &count);
        if (uu1 == temp2 && uu2 == temp2 - 1 && brk) break;
    }
    *k = zz - 1;
    for (zz = (g->cpu_mode ? tempk : imini(tempk, g->nz)) - 1; zz >= 0; --zz) {
        orth_row(o, slice, temp2, zz, apu1, lz, &uu1, &uu2, &brk, &count);
        if (uu1 == temp2 && uu2 == temp2 - 1 && brk) break;
    }
    if (pre_step) *k = ku < 0 ? imaxi(*k, zz) - 1 : imini(*k, zz) + 1;
    return count;
}

/* Traces PET ray r through its tube; *temp = the ray's scale (type 3: 1 / TotV)
 * times the global factor.  Returns 0 when the ray is skipped. */
static int orth_ray(const oracle_geom *g, int64_t r, double *temp, visit_fn vis, void *ctx) {
    v3 s, d;
    load_ray(g, r, &s, &d);
    const double mx = g->bx + (double)g->nx * g->dx;
    const double my = g->by + (double)g->ny * g->dy;
    const double mz = g->bz + (double)g->nz * g->dz;
    v3 diff = {d.x - s.x, d.y - s.y, d.z - s.z};
    if ((diff.x == 0.0 && diff.y == 0.0) || isinf(diff.x) || isinf(diff.y) || isinf(diff.z) || isnan(diff.x) ||
        isnan(diff.y) || isnan(diff.z))
        return 0;
    const double L = sqrt(diff.x * diff.x + diff.y * diff.y + diff.z * diff.z);
    const double r2 = g->orth_width * g->orth_width;
    const double totv = g->cpu_mode ? L * ORTH_PI * r2 : L * (1.0 / ORTH_PI) * r2;
    *temp = (g->proj_type == 3 ? 1.0 / totv : 1.0) * g->global_factor;
    double w[MAXB];
    const int tofon = g->nbins > 1;
    orth_t o;
    o.g = g;
    o.orl = g->proj_type == 2 ? L * g->orth_width : L;
    o.vis = vis;
    o.ctx = ctx;
    o.w = w;
    o.tsum = 1.0;
    int tempk_b = 0;

    if (fabs(diff.z) < 1e-6 && (fabs(diff.y) < 1e-6 || fabs(diff.x) < 1e-6)) {
        const int tk = (int)(fabs(s.z - g->bz) / g->dz);
        if (tk < 0 || tk >= g->nz) return 0;
        int along_x, nrow;
        double b1, d1, d_b, dd, d_db;
        if (fabs(diff.y) < 1e-6 && d.y <= my && d.y >= g->by && s.y <= my && s.y >= g->by) {
            along_x = 1; nrow = g->nx;
            b1 = g->bx; d1 = g->dx; o.b2 = g->by; o.d2 = g->dy;
            d_b = g->by; dd = d.y; d_db = g->dy;
            o.s = s; o.diff = diff;
            o.n1 = g->nx;                        /* kernel d_N1 */
            o.st_slice = 1; o.st_in = g->ny;     /* kernel d_N3, d_N2 */
        } else if (fabs(diff.x) < 1e-6 && d.x <= mx && d.x >= g->bx && s.x <= mx && s.x >= g->bx) {
            along_x = 0; nrow = g->ny;
            b1 = g->by; d1 = g->dy; o.b2 = g->bx; o.d2 = g->dx;
            d_b = g->bx; dd = d.x; d_db = g->dx;
            o.s.x = s.y; o.s.y = s.x; o.s.z = s.z;
            o.diff.x = diff.y; o.diff.y = diff.x; o.diff.z = diff.z;
            o.n1 = g->ny;
            o.st_slice = g->nx; o.st_in = 1;
        } else {
            return 0;
        }
        const int row = perp_start(d_b, dd, d_db, along_x ? g->ny : g->nx);
        const double d_d2 = d1;
        /* the voxels between the end points (projectorType123.cl:541-576); the CPU projector takes the whole row */
        int x1 = 0, x2 = nrow - 1;
        double dT1 = d_d2, dT2 = d_d2;
        if (!g->cpu_mode) {
            const double sa = along_x ? s.x : s.y, da = along_x ? d.x : d.y;
            double dist1, dist2;
            if (sa > da) { dist1 = b1 - da; dist2 = b1 + (double)nrow * d1 - sa; }
            else { dist1 = b1 - sa; dist2 = b1 + (double)nrow * d1 - da; }
            if (dist1 < 0.0) { int kk = (int)ceil(-dist1 / d1); if (kk < nrow) { x1 = kk; dT1 = fmin(dist1 + kk * d1, d1); } }
            if (dist2 > 0.0) { int mm = (int)ceil(dist2 / d1); int kk = nrow - 1 - mm; if (kk >= x1) { x2 = kk; dT2 = fmin(mm * d1 - dist2, d1); } }
        }
        double D = 0.0, ddsign = 0.0;
        if (tofon) { D = (d_d2 * (double)nrow) / copysign(2.0, along_x ? diff.y : diff.x); ddsign = sgn(D); }
        for (int ii = x1; ii <= x2; ++ii) {
            double d_in = d_d2;
            if (x1 > 0 && ii == x1) d_in = dT1;
            else if (x2 < nrow - 1 && ii == x2) d_in = dT2;
            if (tofon) o.tsum = tof_weights(g, ddsign, d_in, D, w);
            orth_slice(&o, ii, b1 + d1 * (double)ii + d1 / 2.0, row, tk, 0, &tempk_b, 0);
            if (tofon) D -= d_d2 * ddsign;
        }
        return 1;
    }

    int ti = 0, tj = 0, tk = 0, ux = 0, uy = 0, uz = 0, xy = 1;
    double txu = 0, tyu = 0, tzu = 0, tc = 0, tx0 = 1e8, ty0 = 1e8, tz0 = 1e8;
    unsigned np = 0;
    int skip;
    if (fabs(diff.z) < 1e-6) {
        tk = (int)(fabs(s.z - g->bz) / g->dz);
        if (tk < 0 || tk >= g->nz) return 0;
        skip = pre2d_xy(g->bx, g->by, diff.x, diff.y, mx, my, g->dx, g->dy, g->nx, g->ny, &ti, &tj, &txu, &tyu, &np,
                        s.x, s.y, d.x, d.y, &tc, &ux, &uy, &tx0, &ty0, &xy);
    } else if (fabs(diff.y) < 1e-6) {
        tj = perp_start(g->by, d.y, g->dy, g->ny);
        skip = pre2d(g->bx, g->bz, diff.x, diff.z, mx, mz, g->dx, g->dz, g->nx, g->nz, &ti, &tk, &txu, &tzu, &np,
                     s.x, s.z, d.x, d.z, &tc, &ux, &uz, &tx0, &tz0);
        xy = 1;
        if (d.y > my || d.y < g->by) skip = 1;
    } else if (fabs(diff.x) < 1e-6) {
        ti = perp_start(g->bx, d.x, g->dx, g->nx);
        skip = pre2d(g->by, g->bz, diff.y, diff.z, my, mz, g->dy, g->dz, g->ny, g->nz, &tj, &tk, &tyu, &tzu, &np,
                     s.y, s.z, d.y, d.z, &tc, &uy, &uz, &ty0, &tz0);
        xy = 0;
        if (d.x > mx || d.x < g->bx) skip = 1;
    } else {
        skip = pre3d(g, mx, my, mz, s, d, diff, &ti, &tj, &tk, &txu, &tyu, &tzu, &np, &tc, &ux, &uy, &uz, &tx0, &ty0,
                     &tz0);
        /* slices along x when the ray is within 45 degrees of the x axis (siddon_pre_loop_3D, ORTH) */
        const double ang = fabs(acos(diff.x / sqrt(diff.x * diff.x + diff.y * diff.y)));
        /* the thresholds are the reference's float literals */
        xy = (ang < (double)0.785398f && ang > 0.0) || (ang > (double)2.35619f && ang < (double)3.92699f) ||
             (ang > (double)5.497787f);
    }
    if (skip) return 0;
    double D = 0.0, ddsign = 0.0;
    if (tofon) {
        double a = diff.x * tc, b = diff.y * tc, c = diff.z * tc;
        D = sqrt(a * a + b * b + c * c) - L / 2.0;
        ddsign = sgn(D);
    }
    double b1, d1;
    int nslice;
    if (!xy) {
        int t; double tt;
        t = ti; ti = tj; tj = t;
        t = ux; ux = uy; uy = t;
        tt = tx0; tx0 = ty0; ty0 = tt;
        tt = txu; txu = tyu; tyu = tt;
        o.s.x = s.y; o.s.y = s.x; o.s.z = s.z;
        o.diff.x = diff.y; o.diff.y = diff.x; o.diff.z = diff.z;
        b1 = g->by; d1 = g->dy; o.b2 = g->bx; o.d2 = g->dx;
        nslice = g->ny; o.n1 = g->nx;
        o.st_slice = g->nx; o.st_in = 1;
    } else {
        o.s = s; o.diff = diff;
        b1 = g->bx; d1 = g->dx; o.b2 = g->by; o.d2 = g->dy;
        nslice = g->nx; o.n1 = g->ny;
        o.st_slice = 1; o.st_in = g->nx;
    }
    const int nsx = xy ? g->nx : g->ny, nsy = xy ? g->ny : g->nx;
    int ti_a = ti, tj_a = tj, tk_a = tk, told = 0;
    double last_ele = 0.0;
    for (unsigned ii = 0; ii < np; ++ii) {
        ti_a = ti; tj_a = tj; tk_a = tk;
        const double tx0_a = tx0, ty0_a = ty0, tz0_a = tz0;
        double *t0, tu;
        int *tijk, u;
        if (tz0 < ty0 && tz0 < tx0) { t0 = &tz0; tu = tzu; tijk = &tk; u = uz; }
        else if (ty0 < tx0) { t0 = &ty0; tu = tyu; tijk = &tj; u = uy; }
        else { t0 = &tx0; tu = txu; tijk = &ti; u = ux; }
        const int pass = (*t0 >= 0.0 && *t0 <= 1.0) || (tc >= 0.0 && tc <= 1.0);
        const double ele = pass ? (fmin(*t0, 1.0) - fmax(tc, 0.0)) * L : 0.0;
        *tijk += u;
        tc = *t0;
        *t0 += tu;
        if (tofon) o.tsum = tof_weights(g, ddsign, ele, D, w);
        if (ii == 0) {
            tempk_b = tk_a;
            if (ux >= 0) {
                for (int kk = ti_a - 1; kk >= 0; --kk)
                    if (orth_slice(&o, kk, b1 + d1 * (double)kk + d1 / 2.0, tj_a, tempk_b, 1, &tempk_b, uz) == 0)
                        break;
            } else {
                for (int kk = ti_a + 1; kk < nslice; ++kk)
                    if (orth_slice(&o, kk, b1 + d1 * (double)kk + d1 / 2.0, tj_a, tempk_b, 1, &tempk_b, uz) == 0)
                        break;
            }
        }
        if (tz0_a >= tx0_a && ty0_a >= tx0_a) {
            orth_slice(&o, ti_a, b1 + d1 * (double)ti_a + d1 / 2.0, tj_a, tk_a, 0, &tempk_b, uz);
            told = ti_a;
        }
        if (tofon) D -= ele * ddsign;
        last_ele = ele;
        if (ti < 0 || ti >= nsx || tj < 0 || tj >= nsy || tk < 0 || tk >= g->nz) break;
    }
    double w2[MAXB];
    if (tofon && g->cpu_mode) {
        tof_weights(g, ddsign, last_ele, D, w2);
        o.w = w2;
    }
    if (ux < 0) {
        if (told != ti_a) ti_a++;
        for (int kk = ti_a - 1; kk >= 0; --kk)
            if (orth_slice(&o, kk, b1 + d1 * (double)kk + d1 / 2.0, tj_a, tk_a, 0, &tempk_b, uz) == 0) break;
    } else {
        if (told != ti_a) ti_a--;
        for (int kk = ti_a + 1; kk < nslice; ++kk)
            if (orth_slice(&o, kk, b1 + d1 * (double)kk + d1 / 2.0, tj_a, tk_a, 0, &tempk_b, uz) == 0) break;
    }
    return 1;
}

/* y[r + to*m_size] = (A img)[r, to] with projector type 2 or 3 (PET). */
int oracle_orth_fp(const oracle_geom *g, const double *img, double *y) {
    if (g->nbins < 1 || g->nbins > MAXB || (g->proj_type != 2 && g->proj_type != 3)) return -1;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t r = 0; r < g->m_size; ++r) {
        fp_ctx f;
        f.img = img;
        f.nb = g->nbins;
        for (int to = 0; to < g->nbins; ++to) f.ax[to] = 0.0;
        double temp = 0.0;
        const int ok = orth_ray(g, r, &temp, fp_visit, &f);
        const double corr = ok ? ray_corr(g, r, 0, 0) : 0.0;
        for (int to = 0; to < g->nbins; ++to) y[r + to * g->m_size] = ok ? f.ax[to] * temp * corr : 0.0;
    }
    return 0;
}

/* img += A^T y, sens += A^T 1 (when not NULL) with projector type 2 or 3.  Serial. */
int oracle_orth_bp(const oracle_geom *g, const double *y, double *img, double *sens) {
    if (g->nbins < 1 || g->nbins > MAXB || (g->proj_type != 2 && g->proj_type != 3)) return -1;
    for (int64_t r = 0; r < g->m_size; ++r) {
        bp_ctx b;
        b.img = img;
        b.sens = sens;
        b.nb = g->nbins;
        int any = sens != NULL;
        for (int to = 0; to < g->nbins; ++to) {
            b.ax[to] = y ? y[r + to * g->m_size] : 0.0;
            any |= b.ax[to] != 0.0;
        }
        if (!any) continue;
        /* the ray's scale is known before the trace: 1 or 1 / TotV, the global factor, the correction */
        v3 s, d;
        load_ray(g, r, &s, &d);
        const double dxl = d.x - s.x, dyl = d.y - s.y, dzl = d.z - s.z;
        const double L = sqrt(dxl * dxl + dyl * dyl + dzl * dzl);
        const double r2 = g->orth_width * g->orth_width;
        const double totv = g->cpu_mode ? L * ORTH_PI * r2 : L * (1.0 / ORTH_PI) * r2;
        b.temp = (g->proj_type == 3 ? 1.0 / totv : 1.0) * g->global_factor * ray_corr(g, r, 0, 0);
        double t;
        orth_ray(g, r, &t, bp_visit, &b);
    }
    return 0;
}
