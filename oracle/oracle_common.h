/*
 * TEST INFRASTRUCTURE ONLY -- shared by the FP64 oracle restatements
 * (siddon_oracle.c, interp_oracle.c): the ray geometry descriptor, ray end
 * points (getDetectorCoordinatesFullSinogram / getDetectorCoordinatesCT and
 * the measurement-level subset mapping getIndex, general_opencl_functions.h:
 * 914-940, 1325-1410, 1601-1628) and the TOF trapezoid weights (TOFDis /
 * TOFWeight / TOFLoop / normPDF, general_opencl_functions.h:1077-1117).
 */
#ifndef OMB_ORACLE_COMMON_H
#define OMB_ORACLE_COMMON_H
#include <math.h>
#include <stdint.h>

typedef struct oracle_geom {
    int modality;            /* 0 PET sinogram, 1 CT panel */
    int nx, ny, nz;
    double dx, dy, dz, bx, by, bz;
    int n_rows, n_cols;
    int64_t proj0, n_proj, m_size;
    int stype, n_subsets, cur_subset;
    double pitch_x, pitch_y;
    double global_factor, epps;
    int nbins;
    double sigma_x;
    const double *tof_centers;
    const float *xy;
    const float *z;
    /* PET corrections (projector_functions.h:1754-1832), NULL when off:
     * multiplicative weight of each of the launch's rays, attenuation image */
    const double *w;
    const double *mu;
    /* modality 3 (index-based events): index pairs of every event */
    const uint16_t *tr;
    const uint16_t *ax;
    /* PET multi-ray: rays per LOR and the crystal sizes they spread over */
    int nr_xy, nr_z;
    double cr_xy, cr_z;
    /* projector types 2 / 3 (orth_oracle part of siddon_oracle.c) */
    int proj_type;          /* 2 orthogonal distance, 3 volume of intersection */
    double orth_width;      /* type 2: tube_width_z; type 3: tube_radius */
    int crystxy, crystz;    /* tube spread transaxially / axially (CRYSTXY / CRYSTZ) */
    double bmin, bmax, vmax;
    const double *V;        /* type 3 volume table, nv entries */
    int nv;
    int cpu_mode;           /* nonzero: the reference CPU projector's variant (see oracle_orth_fp) */
} oracle_geom;


typedef struct { double x, y, z; } v3;

static double sgn(double v) { return (double)((0.0 < v) - (v < 0.0)); }

static void load_ray(const oracle_geom *g, int64_t r, v3 *s, v3 *d) {
    if (g->modality == 2) { /* list-mode events: 6 coordinates each (general_opencl_functions.h:1304-1320) */
        const float *q = g->xy + (g->proj0 + r) * 6;
        s->x = q[0]; s->y = q[1]; s->z = q[2];
        d->x = q[3]; d->y = q[4]; d->z = q[5];
        return;
    }
    if (g->modality == 3) { /* index-based events (general_opencl_functions.h:1277-1301) */
        const int64_t e = (g->proj0 + r) * 2;
        const int t0 = g->tr[e], t1 = g->tr[e + 1], a0 = g->ax[e], a1 = g->ax[e + 1];
        s->x = g->xy[2 * t0]; s->y = g->xy[2 * t0 + 1]; s->z = g->z[a0];
        d->x = g->xy[2 * t1]; d->y = g->xy[2 * t1 + 1]; d->z = g->z[a1];
        return;
    }
    int64_t ix, iy, iz;
    if (g->stype == 0) {
        int64_t nbin = (int64_t)g->n_rows * g->n_cols;
        iz = r / nbin;
        int64_t b = r - iz * nbin;
        iy = b / g->n_rows;
        ix = b - iy * g->n_rows;
        iz += g->proj0;
    } else {
        int64_t S = g->n_subsets, nr = g->n_rows, nc = g->n_cols, x = r;
        if (g->stype == 1) {
            x = x * S + g->cur_subset; iy = x % nc; iz = x / (nr * nc); ix = (x / nc) % nr;
        } else if (g->stype == 2) {
            x = x * S + g->cur_subset; iz = x / (nr * nc); iy = (x / nr) % nc; ix = x % nr;
        } else if (g->stype == 4) {
            x = (x / nr) * nr * S + nr * g->cur_subset + x % nr; iz = x / (nr * nc); iy = (x / nr) % nc; ix = x % nr;
        } else {
            iy = x % nc; x = x / nc * S + g->cur_subset; iz = x / nr; ix = x % nr;
        }
    }
    if (g->modality == 0) {
        const float *q = g->xy + (ix + iy * g->n_rows) * 4;
        s->x = q[0]; s->y = q[1]; s->z = g->z[iz * 2];
        d->x = q[2]; d->y = q[3]; d->z = g->z[iz * 2 + 1];
    } else {
        const float *p = g->xy + iz * 6;
        s->x = p[0]; s->y = p[1]; s->z = p[2];
        d->x = p[3]; d->y = p[4]; d->z = p[5];
        double ux = g->z[iz * 2], uy = g->z[iz * 2 + 1];
        double ia = (double)ix - (double)g->n_rows / 2.0 + 0.5;
        double ib = (double)iy - (double)g->n_cols / 2.0 + 0.5;
        d->x += ia * ux;
        d->y += ia * uy;
        d->z += ib * g->pitch_y;
    }
}

/* Ray lor_z x lor_xy of a multi-ray LOR (multirayCoordinateShiftZ / XY,
 * projector_functions.h:440-461): both end points moved alike. */
static void multiray_shift(const oracle_geom *g, int lor_xy, int lor_z, v3 *s, v3 *d) {
    if (g->nr_z > 1) {
        double iv = g->cr_z / (double)(g->nr_z * 2);
        s->z += iv - g->cr_z / 2.0; d->z += iv - g->cr_z / 2.0;
        iv *= 2.0;
        s->z += iv * lor_z; d->z += iv * lor_z;
    }
    if (g->nr_xy > 1) {
        double iv = g->cr_xy / (double)(g->nr_xy * 2);
        double c = iv - g->cr_xy / 2.0;
        s->x += c; d->x += c; s->y += c; d->y += c;
        iv *= 2.0;
        s->x += iv * lor_xy; d->x += iv * lor_xy; s->y += iv * lor_xy; d->y += iv * lor_xy;
    }
}

#define MAXB 64

static double tof_weights(const oracle_geom *g, double ddsign, double ele, double D, double *w) {
    const double inv = 1.0 / g->sigma_x;
    const double coef = 0.3989422804014327 * inv;
    double dX = ele / 3.0, sdX = dX * ddsign, sum = 0.0;
    for (int to = 0; to < g->nbins; ++to) {
        double c = g->tof_centers[to], a, out;
        a = (D - c) * inv;
        out = coef * exp(-0.5 * a * a);
        for (int tr = 1; tr < 3; ++tr) {
            a = ((D - sdX * (double)tr) - c) * inv;
            out += coef * exp(-0.5 * a * a) * 2.0;
        }
        a = ((D - ele * ddsign) - c) * inv;
        out += coef * exp(-0.5 * a * a);
        w[to] = out * dX;
        sum += w[to];
    }
    if (sum < g->epps) sum = g->epps;
    return sum;
}

#endif
