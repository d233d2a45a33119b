/*
 * TEST INFRASTRUCTURE ONLY -- drivers that run OMEGA's own GPU kernel
 * sources on the CPU, as the pinned oracle of projector types 4 and 5, the
 * TV gradient and the PDHG image update.  Built by oracle/Makefile into
 * oracle/_ref/ (one shared object per kernel variant); nothing in the product
 * loads them.
 *
 * This file is compiled once per variant.  The variant macro selects which
 * reference source is included and which driver is exported; the kernel's
 * own feature macros are the ones omegatomo/projector/init.py:250-442 passes
 * for that case (CUDA, PYTHON, USEGLOBAL, USEIMAGES, USEMAD, TOTLENGTH, CT or
 * PET, FP or BP, PROJ5 / PTYPE4 / BP4 with NVOXELS*, TOF with NBINS) and are
 * given on the compiler's command line by the Makefile.
 *
 *   REFCL_BDD_FP     projectorType5.cl:64-333   projectorType5Forward
 *   REFCL_BDD_BP     projectorType5.cl:381-757  projectorType5Backward (GEOM5)
 *   REFCL_INTERP_FP  projectorType4.cl:84-683   projectorType4Forward (PET or CT, FP)
 *   REFCL_INTERP_BP  projectorType4.cl:84-683   projectorType4Forward (PET, BP, float atomics)
 *   REFCL_INTERP_CTBP projectorType4.cl:718-1100 projectorType4Backward (BP4)
 *   REFCL_AUX        auxKernels.cl:1733-1990    TVKernel (TVGRAD, texture reads)
 *                    auxKernels.cl:2033-2062    PDHGUpdate (PDHG, no subsets)
 *
 * The host-side inputs the reference builds before a launch are restated
 * here so that each kernel receives exactly what the Python projector hands
 * it: the two image summed-area tables (projfunctions.py:203-238), the
 * measurement summed-area table (projfunctions.py:869-878), the per-projection
 * GEOM5 constants (computeGeom5, init.py:6-37) and the texture objects with
 * their filter and addressing modes (projfunctions.py:215-238, 266-290, 969-1003).
 *
 * OMB_REAL = double runs the kernels in FP64 with exact texture weights (the
 * oracle mode); OMB_REAL = float with frac_bits = 8 reproduces the
 * reference's single-precision GPU arithmetic and 8-bit texture weights.
 */
#include "cl_host_shim.h"

#include <stdlib.h>

#include <vector>

#if OMB_FP64
#define float double
#endif
#include "general_opencl_functions.h"
#if defined(REFCL_BDD_FP) || defined(REFCL_BDD_BP)
#include "projectorType5.cl"
#elif defined(REFCL_INTERP_FP) || defined(REFCL_INTERP_BP) || defined(REFCL_INTERP_CTBP)
#include "projectorType4.cl"
#elif defined(REFCL_AUX)
#include "auxKernels.cl"
#endif
#if OMB_FP64
#undef float
#endif

#define REFCL_EXPORT extern "C" __attribute__((visibility("default")))

typedef std::vector<omb_real> rvec;

static rvec to_real(const double *p, size_t n) {
    rvec v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (omb_real)p[i];
    return v;
}

static void from_real(const rvec &v, double *p) {
    for (size_t i = 0; i < v.size(); ++i) p[i] = (double)v[i];
}

static void set_item(unsigned x, unsigned y, unsigned z) {
    blockIdx = make_uint3(x, y, z);
    threadIdx = make_uint3(0, 0, 0);
    blockDim = make_uint3(1, 1, 1);
}

static omb_tex make_tex(const rvec &data, int w, int h, int d, int linear, int normalized, int frac_bits) {
    omb_tex t;
    t.data = data.data();
    t.w = w;
    t.h = h;
    t.d = d;
    t.linear = linear;
    t.normalized = normalized;
    t.frac_bits = frac_bits;
    return t;
}

REFCL_EXPORT int refcl_precision(void) { return (int)sizeof(omb_real); }

#if defined(REFCL_BDD_FP)
/* Forward projection of `n_proj` cone-beam projections.  img: Nx*Ny*Nz,
 * x fastest; xyz: 6 per projection (source, panel centre); uv: 2 per
 * projection; out: n_rows*n_cols*n_proj, rows fastest (accumulated into). */
REFCL_EXPORT int refcl_bdd_fp(int n_rows, int n_cols, double pitch_x, double pitch_y, int nx, int ny, int nz,
                              double bx, double by, double bz, double size_x, double size_y, double dx, double dy,
                              double dz, double scale_x, double scale_y, double scale_z, const double *xyz,
                              const double *uv, long long n_proj, const double *img, int frac_bits, double *out) {
    /* The SAT over (x, z) of every y slice: (Nx+1) x (Nz+1) x Ny, x fastest,
     * node (i, k) = sum of img[a, j, c] for a < i, c < k (projfunctions.py:231-238). */
    const size_t W1 = (size_t)nx + 1, H = (size_t)nz + 1;
    rvec satY(W1 * H * (size_t)ny, (omb_real)0);
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i)
                satY[((size_t)j * H + k + 1) * W1 + i + 1] = (omb_real)img[i + (size_t)nx * (j + (size_t)ny * k)];
    for (int j = 0; j < ny; ++j)       /* cumsum along x (axis 0) */
        for (size_t k = 0; k < H; ++k)
            for (size_t i = 1; i < W1; ++i) satY[((size_t)j * H + k) * W1 + i] += satY[((size_t)j * H + k) * W1 + i - 1];
    for (int j = 0; j < ny; ++j)       /* then along z (axis 1) */
        for (size_t k = 1; k < H; ++k)
            for (size_t i = 0; i < W1; ++i) satY[((size_t)j * H + k) * W1 + i] += satY[((size_t)j * H + k - 1) * W1 + i];
    /* The SAT over (y, z) of every x slice: (Ny+1) x (Nz+1) x Nx, y fastest
     * (projfunctions.py:203-214). */
    const size_t W2 = (size_t)ny + 1;
    rvec satX(W2 * H * (size_t)nx, (omb_real)0);
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                satX[((size_t)i * H + k + 1) * W2 + j + 1] = (omb_real)img[i + (size_t)nx * (j + (size_t)ny * k)];
    for (int i = 0; i < nx; ++i)
        for (size_t k = 0; k < H; ++k)
            for (size_t j = 1; j < W2; ++j) satX[((size_t)i * H + k) * W2 + j] += satX[((size_t)i * H + k) * W2 + j - 1];
    for (int i = 0; i < nx; ++i)
        for (size_t k = 1; k < H; ++k)
            for (size_t j = 0; j < W2; ++j) satX[((size_t)i * H + k) * W2 + j] += satX[((size_t)i * H + k - 1) * W2 + j];
    const omb_tex texY = make_tex(satY, (int)W1, (int)H, ny, 1, 1, frac_bits);
    const omb_tex texX = make_tex(satX, (int)W2, (int)H, nx, 1, 1, frac_bits);
    rvec g = to_real(xyz, (size_t)n_proj * 6), d_uv = to_real(uv, (size_t)n_proj * 2);
    rvec y((size_t)n_rows * n_cols * n_proj, (omb_real)0);
    const int gy = (n_cols + NVOXELSFP - 1) / NVOXELSFP;
#pragma omp parallel for schedule(dynamic)
    for (long long p = 0; p < n_proj; ++p)
        for (int c = 0; c < gy; ++c)
            for (int r = 0; r < n_rows; ++r) {
                set_item((unsigned)r, (unsigned)c, (unsigned)p);
                projectorType5Forward((unsigned)n_rows, (unsigned)n_cols, (omb_real)pitch_x, (omb_real)pitch_y,
                                      (unsigned)nx, (unsigned)ny, (unsigned)nz, (omb_real)bx, (omb_real)by,
                                      (omb_real)bz, (omb_real)size_x, (omb_real)size_y, (omb_real)dx, (omb_real)dy,
                                      (omb_real)dz, (omb_real)scale_x, (omb_real)scale_y, (omb_real)scale_z,
                                      g.data(), d_uv.data(), &texY, &texX, y.data(), n_proj);
            }
    for (size_t i = 0; i < y.size(); ++i) out[i] += (double)y[i];
    return 0;
}
#endif

#if defined(REFCL_BDD_BP)
/* Backprojection of `n_proj` projections into an Nx*Ny*Nz image (x fastest).
 * y: n_rows*n_cols*n_proj, rows fastest.  img and (no_norm == 0) sens are
 * overwritten, as the kernel stores rather than accumulates. */
REFCL_EXPORT int refcl_bdd_bp(int n_rows, int n_cols, double pitch_x, double pitch_y, int nx, int ny, int nz,
                              double bx, double by, double bz, double dx, double dy, double dz, double scale_x,
                              double scale_y, double scale_z, double size_x_bp, double size_z_bp, const double *xyz,
                              const double *uv, long long n_proj, const double *y, int no_norm, int frac_bits,
                              double *img, double *sens) {
    /* computeGeom5 (init.py:6-37): 16 values per projection. */
    rvec geom((size_t)n_proj * 16);
    const omb_real indX = (omb_real)n_rows / (omb_real)2, indY = (omb_real)n_cols / (omb_real)2;
    for (long long p = 0; p < n_proj; ++p) {
        const double *q = xyz + 6 * p;
        const float3 s = make_float3((omb_real)q[0], (omb_real)q[1], (omb_real)q[2]);
        const float3 d = make_float3((omb_real)q[3], (omb_real)q[4], (omb_real)q[5]);
        const float3 apuX = make_float3((omb_real)uv[2 * p] * indX, (omb_real)uv[2 * p + 1] * indX, (omb_real)0);
        const float3 apuY = make_float3((omb_real)0, (omb_real)0, indY * (omb_real)pitch_y);
        const float3 d3 = make_float3(d.x - apuX.x - apuY.x, d.y - apuX.y - apuY.y, d.z - apuX.z - apuY.z);
        const float3 d2 = make_float3(apuX.x - apuY.x, apuX.y - apuY.y, apuX.z - apuY.z);
        const omb_real nX = omb_sqrt(apuX.x * apuX.x + apuX.y * apuX.y + apuX.z * apuX.z);
        const omb_real nY = omb_sqrt(apuY.x * apuY.x + apuY.y * apuY.y + apuY.z * apuY.z);
        const float3 e = make_float3(d3.x - d.x, d3.y - d.y, d3.z - d.z);
        const float3 cp = make_float3(d2.y * e.z - d2.z * e.y, d2.z * e.x - d2.x * e.z, d2.x * e.y - d2.y * e.x);
        const omb_real up = cp.x * (s.x - d.x) + cp.y * (s.y - d.y) + cp.z * (s.z - d.z);
        omb_real *o = geom.data() + 16 * p;
        const omb_real v[16] = {s.x,          s.y,          s.z,          d3.x, d3.y, d3.z, apuX.x / nX, apuX.y / nX,
                                apuX.z / nX, apuY.x / nY, apuY.y / nY, apuY.z / nY, cp.x, cp.y, cp.z, up};
        memcpy(o, v, sizeof(v));
    }
    /* Measurement SAT (projfunctions.py:869-878): (n_rows+1) x (n_cols+1) x
     * n_proj, rows fastest, cumulative along rows then columns. */
    const size_t W = (size_t)n_rows + 1, H = (size_t)n_cols + 1;
    rvec sat(W * H * (size_t)n_proj, (omb_real)0);
    for (long long p = 0; p < n_proj; ++p)
        for (int c = 0; c < n_cols; ++c)
            for (int r = 0; r < n_rows; ++r)
                sat[((size_t)p * H + c + 1) * W + r + 1] = (omb_real)y[r + (size_t)n_rows * (c + (size_t)n_cols * p)];
    for (long long p = 0; p < n_proj; ++p)
        for (size_t c = 0; c < H; ++c)
            for (size_t r = 1; r < W; ++r) sat[((size_t)p * H + c) * W + r] += sat[((size_t)p * H + c) * W + r - 1];
    for (long long p = 0; p < n_proj; ++p)
        for (size_t c = 1; c < H; ++c)
            for (size_t r = 0; r < W; ++r) sat[((size_t)p * H + c) * W + r] += sat[((size_t)p * H + c - 1) * W + r];
    const omb_tex tex = make_tex(sat, (int)W, (int)H, (int)n_proj, 1, 1, frac_bits);
    rvec g = to_real(xyz, (size_t)n_proj * 6), d_uv = to_real(uv, (size_t)n_proj * 2);
    const size_t N = (size_t)nx * ny * nz;
    rvec out(N, (omb_real)0), wsum(N, (omb_real)0);
    const int gz = (nz + NVOXELS5 - 1) / NVOXELS5;
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < gz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                projectorType5Backward((unsigned)n_rows, (unsigned)n_cols, (omb_real)pitch_x, (omb_real)pitch_y,
                                       (unsigned)nx, (unsigned)ny, (unsigned)nz, (omb_real)bx, (omb_real)by,
                                       (omb_real)bz, (omb_real)dx, (omb_real)dy, (omb_real)dz, (omb_real)scale_x,
                                       (omb_real)scale_y, (omb_real)scale_z, (omb_real)size_x_bp,
                                       (omb_real)size_z_bp, g.data(), d_uv.data(), geom.data(), &tex, out.data(),
                                       wsum.data(), (unsigned char)no_norm, n_proj, 0);
            }
    from_real(out, img);
    if (no_norm == 0 && sens) from_real(wsum, sens);
    return 0;
}
#endif

#if defined(REFCL_INTERP_FP) || defined(REFCL_INTERP_BP)
/* Ray-driven type-4 projection of one call: for PET, n_rows x n_cols bins of
 * `n_proj` sinograms (xyz: 4 per bin of the whole sinogram, uv: 2 per
 * sinogram of this call); for CT, n_proj projections (xyz: 6, uv: 2 per
 * projection).  The image is a linear-filtered, normalized, clamp-to-edge
 * texture (projfunctions.py:266-290); bmax = b + N d and the scales
 * dScale4 = 1 / (d N) are passed as the reference passes them.
 * FP: meas (n_rows*n_cols*n_proj*NBINS, bins outermost) is accumulated into.
 * BP: meas is read, img and (no_norm == 0) sens are accumulated into. */
REFCL_EXPORT int refcl_interp(int n_rows, int n_cols, double pitch_x, double pitch_y, double dL, double global_factor,
                              const double *tof_centers, double sigma_x, int nx, int ny, int nz, double bx, double by,
                              double bz, double bmax_x, double bmax_y, double bmax_z, double scale_x, double scale_y,
                              double scale_z, const double *xyz, long long n_xyz, const double *uv, long long n_proj,
                              int frac_bits, double *img, double *meas, double *sens, int no_norm) {
    (void)tof_centers;
    (void)sigma_x;
    (void)sens;
    (void)no_norm;
    (void)frac_bits;
    const size_t N = (size_t)nx * ny * nz;
    const unsigned long long m_size = (unsigned long long)n_rows * n_cols * (unsigned long long)n_proj;
    rvec g = to_real(xyz, (size_t)n_xyz), d_uv = to_real(uv, (size_t)n_proj * 2);
#ifdef TOF
    rvec tc = to_real(tof_centers, NBINS);
#endif
#if defined(REFCL_INTERP_FP)
    rvec im = to_real(img, N);
    const omb_tex tex = make_tex(im, nx, ny, nz, 1, 1, frac_bits);
    rvec y(m_size * NBINS, (omb_real)0);
#define REFCL_IMG_ARG &tex
#define REFCL_OUT_ARG y.data()
#else
    rvec y = to_real(meas, m_size * NBINS);
    rvec out(N, (omb_real)0), wsum(N, (omb_real)0);
#define REFCL_IMG_ARG y.data()
#define REFCL_OUT_ARG out.data()
#endif
#if defined(REFCL_INTERP_FP)
#pragma omp parallel for schedule(dynamic)
#endif
    for (long long p = 0; p < n_proj; ++p)
        for (int c = 0; c < n_cols; ++c)
            for (int r = 0; r < n_rows; ++r) {
                set_item((unsigned)r, (unsigned)c, (unsigned)p);
                projectorType4Forward((unsigned)n_rows, (unsigned)n_cols, (omb_real)pitch_x, (omb_real)pitch_y,
                                      (omb_real)dL, (omb_real)global_factor,
#ifdef TOF
                                      tc.data(), (omb_real)sigma_x,
#endif
                                      (unsigned)nx, (unsigned)ny, (unsigned)nz, (omb_real)bx, (omb_real)by,
                                      (omb_real)bz, (omb_real)bmax_x, (omb_real)bmax_y, (omb_real)bmax_z,
                                      (omb_real)scale_x, (omb_real)scale_y, (omb_real)scale_z, REFCL_IMG_ARG,
                                      REFCL_OUT_ARG, g.data(), d_uv.data(), n_proj,
#if defined(REFCL_INTERP_BP)
                                      wsum.data(),
#endif
                                      (unsigned char)no_norm, m_size, 0u, 0);
            }
#if defined(REFCL_INTERP_FP)
    for (size_t i = 0; i < y.size(); ++i) meas[i] += (double)y[i];
#else
    for (size_t i = 0; i < N; ++i) img[i] += (double)out[i];
    if (no_norm == 0 && sens)
        for (size_t i = 0; i < N; ++i) sens[i] += (double)wsum[i];
#endif
    return 0;
}
#endif

#if defined(REFCL_INTERP_CTBP)
/* Voxel-driven type-4 CT backprojection of n_proj projections: the
 * measurement is a linear-filtered, normalized, clamp-to-edge texture of
 * n_rows x n_cols x n_proj (projfunctions.py:969-980); img and
 * (no_norm == 0) sens are overwritten. */
REFCL_EXPORT int refcl_interp_ct_bp(int n_rows, int n_cols, double pitch_x, double pitch_y, int nx, int ny, int nz,
                                    double bx, double by, double bz, double dx, double dy, double dz, double kerroin,
                                    const double *xyz, const double *uv, long long n_proj, const double *y, int no_norm,
                                    int frac_bits, double *img, double *sens) {
    rvec meas = to_real(y, (size_t)n_rows * n_cols * n_proj);
    const omb_tex tex = make_tex(meas, n_rows, n_cols, (int)n_proj, 1, 1, frac_bits);
    rvec g = to_real(xyz, (size_t)n_proj * 6), d_uv = to_real(uv, (size_t)n_proj * 2);
    const size_t N = (size_t)nx * ny * nz;
    rvec out(N, (omb_real)0), wsum(N, (omb_real)0);
    const int gz = (nz + NVOXELS - 1) / NVOXELS;
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < gz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                projectorType4Backward((unsigned)n_rows, (unsigned)n_cols, (omb_real)pitch_x, (omb_real)pitch_y,
                                       (unsigned)nx, (unsigned)ny, (unsigned)nz, (omb_real)bx, (omb_real)by,
                                       (omb_real)bz, (omb_real)dx, (omb_real)dy, (omb_real)dz, (omb_real)kerroin,
                                       &tex, out.data(), g.data(), d_uv.data(), wsum.data(), (unsigned char)no_norm,
                                       n_proj, 0);
            }
    from_real(out, img);
    if (no_norm == 0 && sens) from_real(wsum, sens);
    return 0;
}
#endif

#if defined(REFCL_AUX)
#if !defined(ANATOMICAL1) && !defined(ANATOMICAL2) && !defined(ANATOMICAL3) && defined(USEIMAGES)
/* TVKernel with texture reads (nearest point, unnormalized, clamp to edge):
 * grad += beta * dTV(u) with smoothing `epps` (the reference's TVsmoothing). */
REFCL_EXPORT int refcl_tv_gradient(int nx, int ny, int nz, const double *u, double sigma, double epps, double beta,
                                   double *grad) {
    const size_t N = (size_t)nx * ny * nz;
    rvec uu = to_real(u, N), g = to_real(grad, N);
    const omb_tex tex = make_tex(uu, nx, ny, nz, 0, 0, 0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                TVKernel(g.data(), &tex, nx, ny, nz, nx, ny, nz, (omb_real)sigma, (omb_real)epps, (omb_real)beta);
            }
    from_real(g, grad);
    return 0;
}
#endif

#if defined(PKMA) || defined(MBSREM) || defined(BSREM)
/* PoissonUpdate (auxKernels.cl:1994-2026) of the variant the build selected, over n voxels (a row). */
REFCL_EXPORT int refcl_poisson(int n, double *im, const double *rhs, double lambda, double epps, double alpha,
                               int positivity) {
    rvec I = to_real(im, (size_t)n), R = to_real(rhs, (size_t)n);
    const int3 Nn = make_int3(n, 1, 1);
    for (int i = 0; i < n; ++i) {
        set_item((unsigned)i, 0u, 0u);
        PoissonUpdate(I.data(), R.data(), Nn, (omb_real)lambda, (omb_real)epps, (omb_real)alpha,
                      (unsigned char)(positivity ? 1 : 0));
    }
    from_real(I, im);
    return 0;
}
#endif

#ifdef PSF
/* Convolution3D_f (auxKernels.cl:190-245): out = the window (2 gx + 1)(2 gy + 1)(2 gz + 1) applied at every
 * voxel with the image mirrored at its faces; the global size is the image size. */
REFCL_EXPORT int refcl_psf(int nx, int ny, int nz, const double *in, const double *w, int gx, int gy, int gz,
                           double *out) {
    const size_t N = (size_t)nx * ny * nz;
    const size_t nw = (size_t)(2 * gx + 1) * (2 * gy + 1) * (2 * gz + 1);
    rvec ii = to_real(in, N), oo((size_t)N, (omb_real)0), ww = to_real(w, nw);
#pragma omp parallel
    {
        gridDim = make_uint3((unsigned)nx, (unsigned)ny, (unsigned)nz);
#pragma omp for schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    set_item((unsigned)i, (unsigned)j, (unsigned)k);
                    Convolution3D_f(ii.data(), oo.data(), ww.data(), gx, gy, gz);
                }
    }
    from_real(oo, out);
    return 0;
}
#endif

#ifdef NLM_
/* The NLM kernel (auxKernels.cl:297-620) in the variant the build selected (NLTYPE, NLMADAPTIVE, NLMREF),
 * search window SWINDOW*, patch PWINDOW*, the images read through the clamp-to-edge texture:
 * grad += beta * g(u).  gauss: the patch weights; uref: the reference image (NLMREF) or NULL. */
REFCL_EXPORT int refcl_nlm(int nx, int ny, int nz, const double *u, const double *gauss, int ng, double h,
                           double epps, double beta, double gamma, double p, double q, double c, double s_adapt,
                           const double *uref, double *grad) {
    const size_t N = (size_t)nx * ny * nz;
    rvec uu = to_real(u, N), g = to_real(grad, N), gg = to_real(gauss, (size_t)ng);
    const omb_tex tex = make_tex(uu, nx, ny, nz, 0, 0, 0);
#ifdef NLMREF
    rvec rr = to_real(uref, N);
    const omb_tex texr = make_tex(rr, nx, ny, nz, 0, 0, 0);
#else
    (void)uref;
#endif
    (void)gamma;
    (void)p;
    (void)q;
    (void)c;
    (void)s_adapt;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                NLM(g.data(), &tex, gg.data(), nx, ny, nz, nx, ny, nz, (omb_real)h, (omb_real)epps, (omb_real)beta
#if NLTYPE >= 3
                    , (omb_real)gamma
#endif
#if NLTYPE == 6
                    , (omb_real)p, (omb_real)q, (omb_real)c
#endif
#ifdef NLMADAPTIVE
                    , (omb_real)s_adapt
#endif
#ifdef NLMREF
                    , &texr
#endif
                );
            }
    from_real(g, grad);
    return 0;
}
#endif

#ifdef GGMRF
/* GGMRFKernel (auxKernels.cl:878-980) over the (2 SWINDOWX + 1)(2 SWINDOWY + 1)(2 SWINDOWZ + 1)
 * neighbourhood: grad += beta * dGGMRF(u), weights w (nw values, centre left out) in the kernel's order.
 * Each work item is its own work group here, so it fills its local cache itself. */
REFCL_EXPORT int refcl_ggmrf(int nx, int ny, int nz, const double *u, const double *w, int nw, double p, double q,
                             double c, double pqc, double beta, double *grad) {
    const size_t N = (size_t)nx * ny * nz;
    rvec uu = to_real(u, N), g = to_real(grad, N), ww = to_real(w, (size_t)nw);
    const omb_tex tex = make_tex(uu, nx, ny, nz, 0, 0, 0);
    const int3 Nn = make_int3(nx, ny, nz);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                GGMRFKernel(g.data(), &tex, ww.data(), Nn, (omb_real)p, (omb_real)q, (omb_real)c, (omb_real)pqc,
                            (omb_real)beta);
            }
    from_real(g, grad);
    return 0;
}
#endif

#ifdef HYPER
/* hyperbolicKernel (auxKernels.cl:1591-1688): grad += beta * dHyperbolic(u) with delta `sigma`. */
REFCL_EXPORT int refcl_hyper(int nx, int ny, int nz, const double *u, const double *w, int nw, double sigma,
                             double epps, double beta, double *grad) {
    const size_t N = (size_t)nx * ny * nz;
    rvec uu = to_real(u, N), g = to_real(grad, N), ww = to_real(w, (size_t)nw);
    const omb_tex tex = make_tex(uu, nx, ny, nz, 0, 0, 0);
    const int3 Nn = make_int3(nx, ny, nz);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                hyperbolicKernel(g.data(), &tex, Nn, Nn, (omb_real)sigma, (omb_real)epps, (omb_real)beta, ww.data());
            }
    from_real(g, grad);
    return 0;
}
#endif

#ifdef RDP
/* RDPKernel (auxKernels.cl:650-875, the 6-neighbour form): grad += beta *
 * dRDP(u); built with USEIMAGES the image is read through the shim's
 * clamp-to-edge texture, without it from the buffer (0 outside). */
REFCL_EXPORT int refcl_rdp(int nx, int ny, int nz, const double *u, double gamma, double epps, double beta,
                           double *grad) {
    const size_t N = (size_t)nx * ny * nz;
    rvec uu = to_real(u, N), g = to_real(grad, N);
#ifdef USEIMAGES
    const omb_tex tex = make_tex(uu, nx, ny, nz, 0, 0, 0);
#endif
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
#ifdef USEIMAGES
                RDPKernel(g.data(), &tex, nx, ny, nz, nx, ny, nz, (omb_real)gamma, (omb_real)epps, (omb_real)beta);
#else
                RDPKernel(g.data(), uu.data(), nx, ny, nz, nx, ny, nz, (omb_real)gamma, (omb_real)epps,
                          (omb_real)beta);
#endif
            }
    from_real(g, grad);
    return 0;
}
#endif

#if defined(PROXTV) && !defined(PROXTGV)
/* One proximal-TV step of the PDHG loop (priors.h:261-281): ProxTVGradient
 * (q += sigma2 * the image differences), ProxTVq (q onto the alpha ball: L2
 * with -DL2, else the max norm), ProxTVDivergence (rhs -= the divergence of
 * q).  q: 3 images (qx, qy, qz), x fastest; updated in place, as is rhs. */
REFCL_EXPORT int refcl_proxtv(int nx, int ny, int nz, const double *im, double *q, double *rhs, double sigma2,
                              double alpha) {
    const size_t N = (size_t)nx * ny * nz;
    rvec I = to_real(im, N), QX = to_real(q, N), QY = to_real(q + N, N), QZ = to_real(q + 2 * N, N);
    rvec R = to_real(rhs, N);
    const int3 Nn = make_int3(nx, ny, nz);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                ProxTVGradient(Nn, Nn, I.data(), QX.data(), QY.data(), QZ.data(), (omb_real)sigma2);
            }
    for (size_t v = 0; v < N; ++v) {
        set_item((unsigned)v, 0u, 0u);
        ProxTVq(QX.data(), QY.data(), QZ.data(), (omb_real)alpha);
    }
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                ProxTVDivergence(Nn, Nn, QX.data(), QY.data(), QZ.data(), R.data());
            }
    from_real(QX, q);
    from_real(QY, q + N);
    from_real(QZ, q + 2 * N);
    from_real(R, rhs);
    return 0;
}
#endif

#if defined(PROXTGV)
/* One proximal TGV step (priors.h:284-313): ProxTVGradient with v, ProxTVq
 * (alpha0), ProxTVDivergence (rhs), ProxTGVSymmDeriv, ProxTGVq (alpha1),
 * ProxTGVDivergence (theta, tau).  q: 3 images; r: 6 (TGVZ) or 3; v: 3 or 2;
 * all updated in place, as is rhs. */
REFCL_EXPORT int refcl_proxtgv(int nx, int ny, int nz, const double *im, double *q, double *r, double *v, double *rhs,
                               double sigma2, double alpha0, double alpha1, double theta, double tau) {
    const size_t N = (size_t)nx * ny * nz;
#if defined(TGVZ)
    const int NR = 6, NV = 3;
#else
    const int NR = 3, NV = 2;
#endif
    rvec I = to_real(im, N), R = to_real(rhs, N);
    rvec Q[3], RR[6], VV[3];
    for (int k = 0; k < 3; ++k) Q[k] = to_real(q + k * N, N);
    for (int k = 0; k < NR; ++k) RR[k] = to_real(r + k * N, N);
    for (int k = 0; k < NV; ++k) VV[k] = to_real(v + k * N, N);
    const int3 Nn = make_int3(nx, ny, nz);
    auto each = [&](auto &&f) {
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    set_item((unsigned)i, (unsigned)j, (unsigned)k);
                    f();
                }
    };
#if defined(TGVZ)
    each([&] { ProxTVGradient(Nn, Nn, I.data(), Q[0].data(), Q[1].data(), Q[2].data(), (omb_real)sigma2,
                              VV[0].data(), VV[1].data(), VV[2].data()); });
#else
    each([&] { ProxTVGradient(Nn, Nn, I.data(), Q[0].data(), Q[1].data(), Q[2].data(), (omb_real)sigma2,
                              VV[0].data(), VV[1].data()); });
#endif
    for (size_t x = 0; x < N; ++x) {
        set_item((unsigned)x, 0u, 0u);
        ProxTVq(Q[0].data(), Q[1].data(), Q[2].data(), (omb_real)alpha0);
    }
    each([&] { ProxTVDivergence(Nn, Nn, Q[0].data(), Q[1].data(), Q[2].data(), R.data()); });
#if defined(TGVZ)
    each([&] { ProxTGVSymmDeriv(Nn, Nn, VV[0].data(), VV[1].data(), VV[2].data(), RR[0].data(), RR[1].data(),
                                RR[2].data(), RR[3].data(), RR[4].data(), RR[5].data(), (omb_real)sigma2); });
    for (size_t x = 0; x < N; ++x) {
        set_item((unsigned)x, 0u, 0u);
        ProxTGVq(RR[0].data(), RR[1].data(), RR[2].data(), RR[3].data(), RR[4].data(), RR[5].data(), (omb_real)alpha1);
    }
    each([&] { ProxTGVDivergence(Nn, Nn, RR[0].data(), RR[1].data(), RR[2].data(), RR[3].data(), RR[4].data(),
                                 RR[5].data(), VV[0].data(), VV[1].data(), VV[2].data(), Q[0].data(), Q[1].data(),
                                 Q[2].data(), (omb_real)theta, (omb_real)tau); });
#else
    each([&] { ProxTGVSymmDeriv(Nn, Nn, VV[0].data(), VV[1].data(), RR[0].data(), RR[1].data(), RR[2].data(),
                                (omb_real)sigma2); });
    for (size_t x = 0; x < N; ++x) {
        set_item((unsigned)x, 0u, 0u);
        ProxTGVq(RR[0].data(), RR[1].data(), RR[2].data(), (omb_real)alpha1);
    }
    each([&] { ProxTGVDivergence(Nn, Nn, RR[0].data(), RR[1].data(), RR[2].data(), VV[0].data(), VV[1].data(),
                                 Q[0].data(), Q[1].data(), Q[2].data(), (omb_real)theta, (omb_real)tau); });
#endif
    for (int k = 0; k < 3; ++k) from_real(Q[k], q + k * N);
    for (int k = 0; k < NR; ++k) from_real(RR[k], r + k * N);
    for (int k = 0; k < NV; ++k) from_real(VV[k], v + k * N);
    from_real(R, rhs);
    return 0;
}
#endif

#ifdef USEIMAGES
/* TVKernel in the variant the build selected (-DSATV, -DTVW1,
 * -DANATOMICAL1/2/3): S is the reference image (or, ANATOMICAL1, the nine
 * tensor channels), C the anatomical weight (options.C, or eta for
 * ANATOMICAL3). */
REFCL_EXPORT int refcl_tv_gradient_ex(int nx, int ny, int nz, const double *u, double sigma, double epps, double beta,
                                      double C, const double *S, double *grad) {
    const size_t N = (size_t)nx * ny * nz;
    rvec uu = to_real(u, N), g = to_real(grad, N);
#if defined(ANATOMICAL1) || defined(ANATOMICAL2) || defined(ANATOMICAL3)
    rvec ss = to_real(S, N * (
#if defined(ANATOMICAL1)
                                  9
#else
                                  1
#endif
                                  ));
#else
    (void)S;
    (void)C;
#endif
    const omb_tex tex = make_tex(uu, nx, ny, nz, 0, 0, 0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                TVKernel(g.data(), &tex, nx, ny, nz, nx, ny, nz, (omb_real)sigma, (omb_real)epps, (omb_real)beta
#if defined(ANATOMICAL2) || defined(ANATOMICAL3)
                         , (omb_real)C
#endif
#if defined(ANATOMICAL1) || defined(ANATOMICAL2) || defined(ANATOMICAL3)
                         , ss.data()
#endif
                );
            }
    from_real(g, grad);
    return 0;
}
#endif

/* PDHGUpdate without subsets: u -= tau * rhs (clamped at epps when
 * positivity is enforced), im = u + theta (u - u_prev). */
REFCL_EXPORT int refcl_pdhg_update(int nx, int ny, int nz, double *im, const double *rhs, double *u, double epps,
                                   double theta, double tau, int positivity) {
    const size_t N = (size_t)nx * ny * nz;
    rvec a = to_real(im, N), r = to_real(rhs, N), b = to_real(u, N);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                set_item((unsigned)i, (unsigned)j, (unsigned)k);
                PDHGUpdate(a.data(), r.data(), b.data(), make_int3(nx, ny, nz), (omb_real)epps, (omb_real)theta,
                           (omb_real)tau, (unsigned char)positivity);
            }
    from_real(a, im);
    from_real(b, u);
    return 0;
}
#endif
