/*
 * TEST INFRASTRUCTURE ONLY -- the FP64 checker for projector type 5
 * (branchless distance-driven).  Nothing in the product links or calls it.
 *
 * Restates OMEGA's GPU kernels source/opencl/projectorType5.cl in double
 * precision, in the reference's own formulation: summed-area tables (SAT,
 * "integral images") sampled with bilinear interpolation and edge clamping,
 * which is what the kernels' linear-filtered, clamp-to-edge textures compute.
 *   forward  projectorType5Forward  projectorType5.cl:64-333 (NVOXELSFP = 8
 *            detector columns per thread, slices along the dominant axis),
 *            detector corners from getDetectorCoordinatesCT
 *            (general_opencl_functions.h:1325-1410, PROJ5 branch), SAT volumes
 *            as omegatomo/projector/projfunctions.py:203-238 builds them;
 *   backward projectorType5Backward projectorType5.cl:381-757 (NVOXELS5 = 1),
 *            per-projection constants as computeGeom5 (omegatomo/projector/
 *            init.py:6-37) derives them, measurement SAT as
 *            projfunctions.py:869-878 builds it.
 * With exact arithmetic the SAT differences equal the footprint integrals;
 * here they are evaluated in FP64 so the result is the reference answer the
 * FP32 GPU kernels are measured against.  One clarification of the
 * reference's "apu != 0" test in the backprojection: a footprint that lies
 * entirely outside the detector counts as zero (the SAT difference is zero
 * in exact arithmetic).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct oracle_ct {
    int nx, ny, nz;
    double dx, dy, dz, bx, by, bz;
    int n_rows, n_cols;
    int64_t proj0, n_proj;   /* projections of this call (global start, count) */
    double pitch_x, pitch_y;
    const float *xy;         /* 6 floats per projection: source, panel centre */
    const float *uv;         /* 2 floats per projection: row direction x pitch_x */
} oracle_ct;

typedef struct { double x, y, z; } d3;

static d3 sub(d3 a, d3 b) { d3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double len3(d3 a) { return sqrt(dot3(a, a)); }
static d3 cross3(d3 a, d3 b) {
    d3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}

/* Bilinear sample of a SAT with (n1+1) x (n2+1) nodes, node (i, k) at
 * sat[k*(n1+1) + i], at continuous node coordinates (e1, e2), clamped. */
static double sat_sample(const double *sat, int n1, int n2, double e1, double e2) {
    if (e1 < 0.0) e1 = 0.0;
    if (e1 > n1) e1 = n1;
    if (e2 < 0.0) e2 = 0.0;
    if (e2 > n2) e2 = n2;
    int i0 = (int)floor(e1), k0 = (int)floor(e2);
    if (i0 > n1) i0 = n1;
    if (k0 > n2) k0 = n2;
    int i1 = i0 < n1 ? i0 + 1 : n1, k1 = k0 < n2 ? k0 + 1 : n2;
    double f1 = e1 - i0, f2 = e2 - k0;
    const int w = n1 + 1;
    return (1 - f1) * (1 - f2) * sat[k0 * w + i0] + f1 * (1 - f2) * sat[k0 * w + i1] +
           (1 - f1) * f2 * sat[k1 * w + i0] + f1 * f2 * sat[k1 * w + i1];
}

/* y[r + c*n_rows + p*n_rows*n_cols] = (A f) for the call's projections. */
int oracle_bdd_fp(const oracle_ct *g, const double *img, double *y) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    /* SAT over (x, z) for every y slice, and over (y, z) for every x slice */
    double *satY = (double *)calloc((size_t)ny * (nx + 1) * (nz + 1), sizeof(double));
    double *satX = (double *)calloc((size_t)nx * (ny + 1) * (nz + 1), sizeof(double));
    if (!satY || !satX) { free(satY); free(satX); return -1; }
    for (int j = 0; j < ny; ++j) {
        double *S = satY + (size_t)j * (nx + 1) * (nz + 1);
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i)
                S[k * (nx + 1) + i] = img[(i - 1) + (size_t)j * nx + (size_t)(k - 1) * nx * ny] +
                                      S[k * (nx + 1) + i - 1] + S[(k - 1) * (nx + 1) + i] -
                                      S[(k - 1) * (nx + 1) + i - 1];
    }
    for (int i = 0; i < nx; ++i) {
        double *S = satX + (size_t)i * (ny + 1) * (nz + 1);
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                S[k * (ny + 1) + j] = img[i + (size_t)(j - 1) * nx + (size_t)(k - 1) * nx * ny] +
                                      S[k * (ny + 1) + j - 1] + S[(k - 1) * (ny + 1) + j] -
                                      S[(k - 1) * (ny + 1) + j - 1];
    }
    const int nr = g->n_rows, nc = g->n_cols, groups = (nc + 7) / 8;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int64_t p = 0; p < g->n_proj; ++p) {
        for (int cg = 0; cg < groups; ++cg) {
            const int64_t gp = g->proj0 + p;
            const float *q = g->xy + gp * 6;
            const d3 s = {q[0], q[1], q[2]};
            const d3 dc = {q[3], q[4], q[5]};
            const double ux = g->uv[gp * 2], uy = g->uv[gp * 2 + 1];
            const int c0 = cg * 8;
            const int maxzz = nc - c0 < 8 ? nc - c0 : 8;
            for (int r = 0; r < nr; ++r) {
                const double ia = (double)r - (double)nr / 2.0 + 0.5;
                const double ib = (double)c0 - (double)nc / 2.0 + 0.5;
                const d3 d = {dc.x + ia * ux, dc.y + ia * uy, dc.z + ib * g->pitch_y};
                const d3 dR = {d.x - 0.5 * ux, d.y - 0.5 * uy, d.z};
                const d3 dL = {d.x + 0.5 * ux, d.y + 0.5 * uy, d.z};
                const d3 dU = {d.x, d.y, d.z + 0.5 * g->pitch_y};
                const d3 dD = {d.x, d.y, d.z - 0.5 * g->pitch_y};
                const d3 dsv = sub(d, s);
                const double L = len3(dsv);
                double kerroin = g->dx * g->dy * g->dz;
                const double apuZ = g->bz - s.z - g->dz / 2.0;
                double temp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                if (fabs(s.x) <= fabs(s.y)) {
                    const double X0 = (dL.x - s.x) / (dL.y - s.y), X1 = (dR.x - s.x) / (dR.y - s.y);
                    const double Z0 = (dU.z - s.z) / (dU.y - s.y), Z1 = (dD.z - s.z) / (dD.y - s.y);
                    kerroin /= fabs(dsv.y / L);
                    const double apuX = g->bx - s.x - g->dx / 2.0, apuV = g->by - s.y;
                    for (int jj = 0; jj < ny; ++jj) {
                        const double v = (jj + 0.5) * g->dy + apuV;
                        const double a0 = v * X0 - apuX, a1 = v * X1 - apuX;
                        const double z0 = v * Z0 - apuZ, z1 = v * Z1 - apuZ;
                        const double xl = fmin(a0, a1), xr = fmax(a0, a1);
                        double zu = fmin(z0, z1), zd = fmax(z0, z1);
                        const double area = fabs((xl - xr) * (zu - zd));
                        const double w = zd - zu;
                        const double *S = satY + (size_t)jj * (nx + 1) * (nz + 1);
                        const double el = xl / g->dx - 0.5, er = xr / g->dx - 0.5;
                        for (int zz = 0; zz < maxzz; ++zz) {
                            const double eu = zu / g->dz - 0.5, ed = zd / g->dz - 0.5;
                            const double A = sat_sample(S, nx, nz, er, eu), B = sat_sample(S, nx, nz, el, ed);
                            const double C = sat_sample(S, nx, nz, er, ed), D = sat_sample(S, nx, nz, el, eu);
                            temp[zz] += (C + D - A - B) / area;
                            zu += w;
                            zd += w;
                        }
                    }
                } else {
                    const double Y0 = (dL.y - s.y) / (dL.x - s.x), Y1 = (dR.y - s.y) / (dR.x - s.x);
                    const double Z0 = (dU.z - s.z) / (dU.x - s.x), Z1 = (dD.z - s.z) / (dD.x - s.x);
                    kerroin /= fabs(dsv.x / L);
                    const double apuY = g->by - s.y - g->dy / 2.0, apuV = g->bx - s.x;
                    for (int ii = 0; ii < nx; ++ii) {
                        const double v = (ii + 0.5) * g->dx + apuV;
                        const double a0 = v * Y0 - apuY, a1 = v * Y1 - apuY;
                        const double z0 = v * Z0 - apuZ, z1 = v * Z1 - apuZ;
                        const double yl = fmin(a0, a1), yr = fmax(a0, a1);
                        double zu = fmin(z0, z1), zd = fmax(z0, z1);
                        const double area = fabs((yl - yr) * (zu - zd));
                        const double w = zd - zu;
                        const double *S = satX + (size_t)ii * (ny + 1) * (nz + 1);
                        const double el = yl / g->dy - 0.5, er = yr / g->dy - 0.5;
                        for (int zz = 0; zz < maxzz; ++zz) {
                            const double eu = zu / g->dz - 0.5, ed = zd / g->dz - 0.5;
                            const double A = sat_sample(S, ny, nz, er, eu), B = sat_sample(S, ny, nz, el, ed);
                            const double C = sat_sample(S, ny, nz, er, ed), D = sat_sample(S, ny, nz, el, eu);
                            temp[zz] += (C + D - A - B) / area;
                            zu += w;
                            zd += w;
                        }
                    }
                }
                int64_t idx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
                for (int zz = 0; zz < maxzz; ++zz, idx += nr) y[idx] = temp[zz] * kerroin;
            }
        }
    }
    free(satY);
    free(satX);
    return 0;
}

/* img = A^T y (voxel driven), sens = sum of weights where the footprint has
 * a nonzero integral (when sens is not NULL). */
int oracle_bdd_bp(const oracle_ct *g, const double *y, double *img, double *sens) {
    const int nr = g->n_rows, nc = g->n_cols;
    const int64_t np = g->n_proj;
    double *sat = (double *)calloc((size_t)np * (nr + 1) * (nc + 1), sizeof(double));
    if (!sat) return -1;
    for (int64_t p = 0; p < np; ++p) {
        double *S = sat + (size_t)p * (nr + 1) * (nc + 1);
        const double *yp = y + p * (int64_t)nr * nc;
        for (int c = 1; c <= nc; ++c)
            for (int r = 1; r <= nr; ++r)
                S[c * (nr + 1) + r] = yp[(r - 1) + (int64_t)(c - 1) * nr] + S[c * (nr + 1) + r - 1] +
                                      S[(c - 1) * (nr + 1) + r] - S[(c - 1) * (nr + 1) + r - 1];
    }
    const int nx = g->nx, ny = g->ny, nz = g->nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k) {
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                const d3 dV = {i * g->dx + g->dx / 2.0 + g->bx, j * g->dy + g->dy / 2.0 + g->by,
                               k * g->dz + g->dz / 2.0 + g->bz};
                double temp = 0.0, wsum = 0.0;
                for (int64_t p = 0; p < np; ++p) {
                    const int64_t gp = g->proj0 + p;
                    const float *q = g->xy + gp * 6;
                    const d3 s = {q[0], q[1], q[2]};
                    const d3 d = {q[3], q[4], q[5]};
                    const double ix = (double)nr / 2.0, iy = (double)nc / 2.0;
                    const d3 apuX = {g->uv[gp * 2] * ix, g->uv[gp * 2 + 1] * ix, 0.0};
                    const d3 apuY = {0.0, 0.0, iy * g->pitch_y};
                    const d3 dd2 = sub(apuX, apuY);
                    const d3 dd3 = sub(sub(d, apuX), apuY);
                    const double lx = len3(apuX), ly = len3(apuY);
                    const d3 normX = {apuX.x / lx, apuX.y / lx, apuX.z / lx};
                    const d3 normY = {apuY.x / ly, apuY.y / ly, apuY.z / ly};
                    const d3 cP = cross3(dd2, sub(dd3, d));
                    const double upper = dot3(cP, sub(s, d));
                    const int sxdim = fabs(s.x) <= fabs(s.y);
                    d3 cLU, cRD;
                    if (sxdim) {
                        if (s.y > 0.0) {
                            cLU.x = dV.x - g->dx / 2.0; cLU.y = dV.y; cLU.z = dV.z - g->dz / 2.0;
                            cRD.x = dV.x + g->dx / 2.0; cRD.y = dV.y; cRD.z = dV.z + g->dz / 2.0;
                        } else {
                            cLU.x = dV.x + g->dx / 2.0; cLU.y = dV.y; cLU.z = dV.z - g->dz / 2.0;
                            cRD.x = dV.x - g->dx / 2.0; cRD.y = dV.y; cRD.z = dV.z + g->dz / 2.0;
                        }
                    } else {
                        if (s.x > 0.0) {
                            cLU.x = dV.x; cLU.y = dV.y + g->dy / 2.0; cLU.z = dV.z - g->dz / 2.0;
                            cRD.x = dV.x; cRD.y = dV.y - g->dy / 2.0; cRD.z = dV.z + g->dz / 2.0;
                        } else {
                            cLU.x = dV.x; cLU.y = dV.y - g->dy / 2.0; cLU.z = dV.z - g->dz / 2.0;
                            cRD.x = dV.x; cRD.y = dV.y + g->dy / 2.0; cRD.z = dV.z + g->dz / 2.0;
                        }
                    }
                    const d3 vLU = sub(cLU, s), vRD = sub(cRD, s);
                    const double tLU = upper / (-dot3(vLU, cP)), tRD = upper / (-dot3(vRD, cP));
                    const d3 pLU = {vLU.x * tLU + s.x - dd3.x, vLU.y * tLU + s.y - dd3.y, vLU.z * tLU + s.z - dd3.z};
                    const d3 pRD = {vRD.x * tRD + s.x - dd3.x, vRD.y * tRD + s.y - dd3.y, vRD.z * tRD + s.z - dd3.z};
                    double Ax = dot3(pLU, normX) + g->pitch_x / 2.0, Ay = dot3(pLU, normY) + g->pitch_y / 2.0;
                    double Dx = dot3(pRD, normX) + g->pitch_x / 2.0, Dy = dot3(pRD, normY) + g->pitch_y / 2.0;
                    if (Dx > Ax) { double t = Ax; Ax = Dx; Dx = t; }
                    if (Dy > Ay) { double t = Ay; Ay = Dy; Dy = t; }
                    /* continuous pixel-edge coordinates of the footprint */
                    const double ea = Ax / g->pitch_x - 0.5, ed = Dx / g->pitch_x - 0.5;
                    const double fa = Ay / g->pitch_y - 0.5, fd = Dy / g->pitch_y - 0.5;
                    double apu = 0.0;
                    const double cxl = fmax(ed, 0.0), cxr = fmin(ea, (double)nr);
                    const double cyl = fmax(fd, 0.0), cyr = fmin(fa, (double)nc);
                    if (cxr > cxl && cyr > cyl) {
                        const double *S = sat + (size_t)p * (nr + 1) * (nc + 1);
                        const double A = sat_sample(S, nr, nc, ea, fa), B = sat_sample(S, nr, nc, ea, fd);
                        const double C = sat_sample(S, nr, nc, ed, fa), D = sat_sample(S, nr, nc, ed, fd);
                        apu = A + D - C - B;
                    }
                    const d3 vd = sub(dV, s);
                    const double ker = sxdim ? g->dy * len3(vd) / fabs(vd.y) : g->dx * len3(vd) / fabs(vd.x);
                    if (apu != 0.0) {
                        temp += apu * ker;
                        wsum += ker;
                    }
                }
                const int64_t n = i + (int64_t)j * nx + (int64_t)k * nx * ny;
                img[n] = temp;
                if (sens) sens[n] = wsum;
            }
        }
    }
    free(sat);
    return 0;
}

/* Ray-driven (scatter) backprojection: the exact adjoint of oracle_bdd_fp.
 * Every ray's forward weight kerroin / area times the clamped overlap of its
 * footprint with voxel (i, k) of slice jj -- the quantity the summed-area
 * difference integrates -- carries y[ray] back onto that voxel.  The
 * 8-column groups share their first column's geometry exactly as in the
 * forward projection (projectorType5.cl:166-174).  img is overwritten;
 * sens (when not NULL) receives A^T 1. */
static double overlap(double a, double b, double lo, double hi) {
    const double l = a > lo ? a : lo, h = b < hi ? b : hi;
    return h > l ? h - l : 0.0;
}

int oracle_bdd_bp_ray(const oracle_ct *g, const double *y, double *img, double *sens) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t N = (size_t)nx * ny * nz;
    for (size_t n = 0; n < N; ++n) {
        img[n] = 0.0;
        if (sens) sens[n] = 0.0;
    }
    const int nr = g->n_rows, nc = g->n_cols, groups = (nc + 7) / 8;
    for (int64_t p = 0; p < g->n_proj; ++p) {
        for (int cg = 0; cg < groups; ++cg) {
            const int64_t gp = g->proj0 + p;
            const float *q = g->xy + gp * 6;
            const d3 s = {q[0], q[1], q[2]};
            const d3 dc = {q[3], q[4], q[5]};
            const double ux = g->uv[gp * 2], uy = g->uv[gp * 2 + 1];
            const int c0 = cg * 8;
            const int maxzz = nc - c0 < 8 ? nc - c0 : 8;
            for (int r = 0; r < nr; ++r) {
                const double ia = (double)r - (double)nr / 2.0 + 0.5;
                const double ib = (double)c0 - (double)nc / 2.0 + 0.5;
                const d3 d = {dc.x + ia * ux, dc.y + ia * uy, dc.z + ib * g->pitch_y};
                const d3 dR = {d.x - 0.5 * ux, d.y - 0.5 * uy, d.z};
                const d3 dL = {d.x + 0.5 * ux, d.y + 0.5 * uy, d.z};
                const d3 dU = {d.x, d.y, d.z + 0.5 * g->pitch_y};
                const d3 dD = {d.x, d.y, d.z - 0.5 * g->pitch_y};
                const d3 dsv = sub(d, s);
                const double L = len3(dsv);
                double kerroin = g->dx * g->dy * g->dz;
                const double apuZ = g->bz - s.z - g->dz / 2.0;
                const int ysl = fabs(s.x) <= fabs(s.y);
                double P0, P1, Z0, Z1, apuL, apuV, dlat, dsl;
                int nsl, nlat;
                if (ysl) {
                    P0 = (dL.x - s.x) / (dL.y - s.y); P1 = (dR.x - s.x) / (dR.y - s.y);
                    Z0 = (dU.z - s.z) / (dU.y - s.y); Z1 = (dD.z - s.z) / (dD.y - s.y);
                    kerroin /= fabs(dsv.y / L);
                    apuL = g->bx - s.x - g->dx / 2.0; apuV = g->by - s.y;
                    dlat = g->dx; dsl = g->dy; nsl = ny; nlat = nx;
                } else {
                    P0 = (dL.y - s.y) / (dL.x - s.x); P1 = (dR.y - s.y) / (dR.x - s.x);
                    Z0 = (dU.z - s.z) / (dU.x - s.x); Z1 = (dD.z - s.z) / (dD.x - s.x);
                    kerroin /= fabs(dsv.x / L);
                    apuL = g->by - s.y - g->dy / 2.0; apuV = g->bx - s.x;
                    dlat = g->dy; dsl = g->dx; nsl = nx; nlat = ny;
                }
                const int64_t yidx = r + (int64_t)c0 * nr + p * (int64_t)nr * nc;
                for (int jj = 0; jj < nsl; ++jj) {
                    const double v = (jj + 0.5) * dsl + apuV;
                    const double a0 = v * P0 - apuL, a1 = v * P1 - apuL;
                    const double z0 = v * Z0 - apuZ, z1 = v * Z1 - apuZ;
                    const double xl = fmin(a0, a1), xr = fmax(a0, a1);
                    const double zu = fmin(z0, z1), zd = fmax(z0, z1);
                    const double area = fabs((xl - xr) * (zu - zd));
                    const double w = zd - zu;
                    /* voxel-edge coordinates of the footprint */
                    const double el = xl / dlat - 0.5, er = xr / dlat - 0.5;
                    const int ia0 = (int)floor(fmax(el, 0.0)), ia1 = (int)ceil(fmin(er, (double)nlat));
                    for (int zz = 0; zz < maxzz; ++zz) {
                        const double yv = y[yidx + (int64_t)zz * nr];
                        const double eu = (zu + zz * w) / g->dz - 0.5, ed = (zd + zz * w) / g->dz - 0.5;
                        const int k0 = (int)floor(fmax(eu, 0.0)), k1 = (int)ceil(fmin(ed, (double)nz));
                        for (int k = k0; k < k1; ++k) {
                            const double oz = overlap(eu, ed, (double)k, (double)k + 1.0);
                            if (oz <= 0.0) continue;
                            for (int i = ia0; i < ia1; ++i) {
                                const double ox = overlap(el, er, (double)i, (double)i + 1.0);
                                if (ox <= 0.0) continue;
                                const double wt = kerroin * ox * oz / area;
                                const size_t n = ysl ? (size_t)i + (size_t)jj * nx + (size_t)k * nx * ny
                                                     : (size_t)jj + (size_t)i * nx + (size_t)k * nx * ny;
                                img[n] += wt * yv;
                                if (sens) sens[n] += wt;
                            }
                        }
                    }
                }
            }
        }
    }
    return 0;
}
