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

static int pre2d(double b1, double b2, double diff1, double diff2, double max1, double max2, double d1, double d2,
                 int n1, int n2, int *t1, int *t2, double *t1u, double *t2u, unsigned *np, double xs, double ys,
                 double xd, double yd, double *tc, int *u1, int *u2, double *t10, double *t20) {
    double apx = b1 - xs, apy = b2 - ys;
    *t10 = apx / diff1;
    *t20 = apy / diff2;
    double txb = (max1 - xs) / diff1, tyb = (max2 - ys) / diff2;
    double txmin = fmin(*t10, txb), txmax = fmax(*t10, txb), tymin = fmin(*t20, tyb), tymax = fmax(*t20, tyb);
    *tc = fmax(txmin, tymin);
    double tmax = fmin(txmax, tymax);
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
