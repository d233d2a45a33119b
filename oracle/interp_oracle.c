/*
 * TEST INFRASTRUCTURE ONLY -- the FP64 checker for projector type 4
 * (interpolation-based).  Nothing in the product links or calls it.
 *
 * Restates OMEGA's GPU kernels source/opencl/projectorType4.cl in double
 * precision, with exact trilinear / bilinear interpolation in place of the
 * kernels' linear-filtered, clamp-to-edge textures (whose weights carry 8
 * fractional bits):
 *   forward   projectorType4Forward, non-Joseph branch (the Python front end
 *             never defines JOSEPH): t-range against [b, bmax] (392-401),
 *             tStep = dL / L, nSteps = floor((tEnd - tStart) / tStep) + 1
 *             (467-476), samples at tStart + n tStep, texture coordinate
 *             (p - b) / d - 1/2 (normalised coordinate times N minus one half),
 *             PET output scaled by global_factor / L (TOTLENGTH), CT output the
 *             plain sum (forwardProjectAF, general_opencl_functions.h:
 *             1961-1967); TOF with TOFLoop / denominator (1103-1207);
 *   backward  (PET) the same march, weight dL * global_factor / L times y (or
 *             the TOF-weighted sum of rhs, 1212-1275) added to the voxel
 *             floor(p / d) per axis, flat index 0 and indices >= N skipped,
 *             and the TOF distance advanced only after a kept sample
 *             (projectorType4.cl:579-604);
 *   backward  (CT) projectorType4Backward (718-1100): voxel centre projected
 *             from the source onto the panel plane, bilinear sample of the
 *             projection where 0 <= px, py <= 1, weight L^3 / |v|^2 * kerroin,
 *             sensitivity summed where the sample is nonzero.
 * The sample count uses the same separately rounded double operations as the
 * GPU set-up, so both take the same number of samples.  bmax is float32
 * (b + N d), as the reference's host code passes it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "oracle_common.h"

typedef struct oracle_ct4 {
    int nx, ny, nz;
    double dx, dy, dz, bx, by, bz;
    int n_rows, n_cols;
    int64_t proj0, n_proj;
    double pitch_x, pitch_y;
    const float *xy;         /* 6 floats per projection: source, panel centre */
    const float *uv;         /* 2 floats per projection: row direction x pitch_x */
} oracle_ct4;

static double upper_edge(double b, int n, double d) { return (double)(float)(b + (double)n * d); }

/* Ray set-up; returns the sample count (0: the ray misses the FOV). */
static unsigned march(const oracle_geom *g, v3 s, v3 d, double dL, double *ts, double *tstep, double *L) {
    const double vx = d.x - s.x, vy = d.y - s.y, vz = d.z - s.z;
    const double t0x = (g->bx - s.x) / vx, t1x = (upper_edge(g->bx, g->nx, g->dx) - s.x) / vx;
    const double t0y = (g->by - s.y) / vy, t1y = (upper_edge(g->by, g->ny, g->dy) - s.y) / vy;
    const double t0z = (g->bz - s.z) / vz, t1z = (upper_edge(g->bz, g->nz, g->dz) - s.z) / vz;
    const double tstart = fmax(fmax(fmin(t0x, t1x), fmin(t0y, t1y)), fmin(t0z, t1z));
    const double tend = fmin(fmin(fmax(t0x, t1x), fmax(t0y, t1y)), fmax(t0z, t1z));
    if (!(tstart < tend)) return 0;
    const double vxx = vx * vx, vyy = vy * vy, vzz = vz * vz;
    *L = sqrt((vxx + vyy) + vzz);
    *tstep = dL / *L;
    const double q = (tend - tstart) / *tstep;
    if (!(q >= 0.0) || q >= 4.0e9) return 0;
    *ts = tstart;
    return (unsigned)q + 1u;
}

static double trilinear(const oracle_geom *g, const double *img, double x, double y, double z) {
    if (x < -1.0) x = -1.0;
    if (x > g->nx) x = g->nx;
    if (y < -1.0) y = -1.0;
    if (y > g->ny) y = g->ny;
    if (z < -1.0) z = -1.0;
    if (z > g->nz) z = g->nz;
    const double fx = floor(x), fy = floor(y), fz = floor(z);
    const double ax = x - fx, ay = y - fy, az = z - fz;
    int xi[2] = {(int)fx, (int)fx + 1}, yi[2] = {(int)fy, (int)fy + 1}, zi[2] = {(int)fz, (int)fz + 1};
    for (int k = 0; k < 2; ++k) {
        xi[k] = xi[k] < 0 ? 0 : (xi[k] >= g->nx ? g->nx - 1 : xi[k]);
        yi[k] = yi[k] < 0 ? 0 : (yi[k] >= g->ny ? g->ny - 1 : yi[k]);
        zi[k] = zi[k] < 0 ? 0 : (zi[k] >= g->nz ? g->nz - 1 : zi[k]);
    }
    const double wx[2] = {1.0 - ax, ax}, wy[2] = {1.0 - ay, ay}, wz[2] = {1.0 - az, az};
    double out = 0.0;
    for (int c = 0; c < 2; ++c)
        for (int b = 0; b < 2; ++b)
            for (int a = 0; a < 2; ++a)
                out += wx[a] * wy[b] * wz[c] *
                       img[xi[a] + (int64_t)yi[b] * g->nx + (int64_t)zi[c] * g->nx * g->ny];
    return out;
}

/* y[r + bin * m_size] = (A f), A the type-4 forward projector. */
int oracle_interp_fp(const oracle_geom *g, double dL, const double *img, double *y) {
    const int nb = g->nbins;
    if (nb > MAXB) return -1;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < g->m_size; ++r) {
        double ax[MAXB], w[MAXB];
        for (int to = 0; to < nb; ++to) ax[to] = 0.0;
        v3 s, d;
        load_ray(g, r, &s, &d);
        double ts = 0.0, tstep = 0.0, L = 0.0;
        const unsigned n = march(g, s, d, dL, &ts, &tstep, &L);
        const double vx = d.x - s.x, vy = d.y - s.y, vz = d.z - s.z;
        const double D0 = fabs(ts) * L - 0.5 * L, ddsign = sgn(D0);
        for (unsigned ii = 0; ii < n; ++ii) {
            const double t = ts + (double)ii * tstep;
            const double px = (s.x + vx * t - g->bx) / g->dx - 0.5;
            const double py = (s.y + vy * t - g->by) / g->dy - 0.5;
            const double pz = (s.z + vz * t - g->bz) / g->dz - 0.5;
            const double val = dL * trilinear(g, img, px, py, pz);
            if (nb == 1) {
                ax[0] += val;
            } else {
                const double D = D0 - (double)ii * dL * ddsign;
                const double tsum = tof_weights(g, ddsign, dL, D, w);
                for (int to = 0; to < nb; ++to) ax[to] += w[to] * (val / tsum);
            }
        }
        const double temp = n == 0 ? 0.0 : (g->modality != 1 ? g->global_factor / L : 1.0);
        for (int to = 0; to < nb; ++to) y[r + (int64_t)to * g->m_size] = ax[to] * temp;
    }
    return 0;
}

/* img += A^T y (PET, ray driven), sens += A^T 1 when sens != NULL; y == NULL
 * backprojects ones.  Serial over rays (no atomics needed). */
int oracle_interp_bp(const oracle_geom *g, double dL, const double *y, double *img, double *sens) {
    const int nb = g->nbins;
    if (nb > MAXB) return -1;
    const uint64_t nx = (uint64_t)g->nx, nxy = nx * (uint64_t)g->ny, ntot = nxy * (uint64_t)g->nz;
    const double ivx = 1.0 / g->dx, ivy = 1.0 / g->dy, ivz = 1.0 / g->dz;
    for (int64_t r = 0; r < g->m_size; ++r) {
        double ax[MAXB], w[MAXB];
        for (int to = 0; to < nb; ++to) ax[to] = y ? y[r + (int64_t)to * g->m_size] : 1.0;
        v3 s, d;
        load_ray(g, r, &s, &d);
        double ts = 0.0, tstep = 0.0, L = 0.0;
        const unsigned n = march(g, s, d, dL, &ts, &tstep, &L);
        if (n == 0) continue;
        const double vx = d.x - s.x, vy = d.y - s.y, vz = d.z - s.z;
        const double le = dL * (g->global_factor / L);
        const double D0 = fabs(ts) * L - 0.5 * L, ddsign = sgn(D0);
        unsigned kept = 0;
        for (unsigned ii = 0; ii < n; ++ii) {
            const double t = ts + (double)ii * tstep;
            /* the same separately rounded operations as the GPU kernel: on
             * voxel faces both pick the same neighbour */
            const double px = ((s.x + vx * t) - g->bx) * ivx;
            const double py = ((s.y + vy * t) - g->by) * ivy;
            const double pz = ((s.z + vz * t) - g->bz) * ivz;
            const uint64_t ux = px > 0.0 ? (uint64_t)px : 0, uy = py > 0.0 ? (uint64_t)py : 0,
                           uz = pz > 0.0 ? (uint64_t)pz : 0;
            const uint64_t ind = ux + uy * nx + uz * nxy;
            double yax, val;
            if (nb == 1) {
                yax = ax[0] * le;
                val = le;
            } else {
                const double D = D0 - (double)kept * dL * ddsign;
                const double tsum = tof_weights(g, ddsign, dL, D, w);
                yax = 0.0;
                val = 0.0;
                for (int to = 0; to < nb; ++to) {
                    const double a = le / tsum * w[to];
                    val += a;
                    yax += a * ax[to];
                }
            }
            if (ind == 0 || ind >= ntot) continue;
            ++kept;
            if (img) img[ind] += yax;
            if (sens) sens[ind] += val;
        }
    }
    return 0;
}

/* Voxel-driven CT backprojection: img = A^T y, sens = the weight sums. */
int oracle_interp_ct_bp(const oracle_ct4 *g, double kerroin, const double *y, double *img, double *sens) {
    const int nr = g->n_rows, nc = g->n_cols;
    const double kox = nr * g->pitch_x, koy = nc * g->pitch_y;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const double qx = (i + 0.5) * g->dx + g->bx, qy = (j + 0.5) * g->dy + g->by,
                             qz = (k + 0.5) * g->dz + g->bz;
                double acc = 0.0, wsum = 0.0;
                for (int64_t p = 0; p < g->n_proj; ++p) {
                    const int64_t gp = g->proj0 + p;
                    const float *q = g->xy + gp * 6;
                    const double sx = q[0], sy = q[1], sz = q[2], d1x = q[3], d1y = q[4], d1z = q[5];
                    const double ux = g->uv[gp * 2], uy = g->uv[gp * 2 + 1];
                    /* apuX = (nr/2) (ux, uy, 0), apuY = (0, 0, (nc/2) pitch_y) */
                    const double ax_ = 0.5 * nr * ux, ay_ = 0.5 * nr * uy, az_ = 0.5 * nc * g->pitch_y;
                    const double d3x = d1x - ax_, d3y = d1y - ay_, d3z = d1z - az_;
                    /* cP = cross(apuX - apuY, -apuX - apuY) */
                    const double e1x = ax_, e1y = ay_, e1z = -az_, e2x = -ax_, e2y = -ay_, e2z = -az_;
                    const double cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
                    const double vx = qx - sx, vy = qy - sy, vz = qz - sz;
                    const double t = (cx * (d1x - sx) + cy * (d1y - sy) + cz * (d1z - sz)) / (cx * vx + cy * vy + cz * vz);
                    const double hx = sx + vx * t, hy = sy + vy * t, hz = sz + vz * t;
                    const double L = sqrt((hx - sx) * (hx - sx) + (hy - sy) * (hy - sy) + (hz - sz) * (hz - sz));
                    const double l1 = vx * vx + vy * vy + vz * vz;
                    const double weight = L * L * L / l1 * kerroin;
                    const double lx = sqrt(ax_ * ax_ + ay_ * ay_);
                    const double px = ((hx - d3x) * ax_ / lx + (hy - d3y) * ay_ / lx) / kox;
                    const double py = (hz - d3z) / koy;
                    if (!(px >= 0.0 && px <= 1.0 && py >= 0.0 && py <= 1.0)) continue;
                    /* bilinear, clamp to edge, texel coordinates px*nr - 1/2, py*nc - 1/2 */
                    const double u = px * nr - 0.5, v = py * nc - 0.5;
                    const double fu = floor(u), fv = floor(v);
                    const double au = u - fu, av = v - fv;
                    int u0 = (int)fu, u1 = u0 + 1, v0 = (int)fv, v1 = v0 + 1;
                    u0 = u0 < 0 ? 0 : (u0 >= nr ? nr - 1 : u0);
                    u1 = u1 < 0 ? 0 : (u1 >= nr ? nr - 1 : u1);
                    v0 = v0 < 0 ? 0 : (v0 >= nc ? nc - 1 : v0);
                    v1 = v1 < 0 ? 0 : (v1 >= nc ? nc - 1 : v1);
                    const double *yp = y + p * (int64_t)nr * nc;
                    const double yv = (1 - au) * (1 - av) * yp[u0 + (int64_t)v0 * nr] + au * (1 - av) * yp[u1 + (int64_t)v0 * nr] +
                                      (1 - au) * av * yp[u0 + (int64_t)v1 * nr] + au * av * yp[u1 + (int64_t)v1 * nr];
                    if (yv != 0.0) {
                        acc += yv * weight;
                        wsum += weight;
                    }
                }
                const int64_t n = i + (int64_t)j * g->nx + (int64_t)k * g->nx * g->ny;
                img[n] = acc;
                if (sens) sens[n] = wsum;
            }
        }
    }
    return 0;
}
