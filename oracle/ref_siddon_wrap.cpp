/*
 * TEST INFRASTRUCTURE ONLY.  Thin C entry points around OMEGA's own OpenMP
 * CPU projector, projectorType123Implementation4<T>
 * (source/cpp/projector_functions.h:1312), compiled from the reference
 * sources where they lie (oracle/Makefile passes -I to them); nothing of the
 * reference is copied here.  Output goes to oracle/_ref/libref_siddon.so.
 * Used to pin the FP64 restatement (oracle/siddon_oracle.c) against the
 * reference itself, and as the timed CPU baseline of bench.py; also the
 * reference's CPU non-local means gradient (NLM.h), which pins
 * oracle/image_oracle.py's restatement.
 *
 * PET sinogram data, whole-sinogram subsets: the caller passes the z pairs of
 * the sinograms to project, so the function runs with subsets = 1.
 */
#include <cstdint>

#include "projector_functions.h"
#include "NLM.h"
#include "MRP.h"

template <typename T>
static int run(int fp, uint32_t nx, uint32_t ny, uint32_t nz, T dx, T dy, T dz, T bx, T by, T bz, uint32_t n_rows,
               uint32_t n_cols, uint32_t n_proj, const T *xy, const T *z, T *input, T *output, T *sens, uint32_t nbins,
               T sigma_x, T *tof_centers, T global_factor, T epps, uint32_t n_threads, T *norm = nullptr,
               T *atten = nullptr, int ct_atten = 1, T *scat = nullptr, uint16_t n_rays_xy = 1,
               uint16_t n_rays_z = 1, T cr_xy = 0, T cr_z = 0) {
    paramStruct<T> p;
    p.subsetType = 8;
    p.subsets = 1;
    p.currentSubset = 0;
    p.size_x = n_rows;
    p.size_y = n_cols;
    p.dx = dx; p.dy = dy; p.dz = dz;
    p.Nx = nx; p.Ny = ny; p.Nz = nz;
    p.bx = bx; p.by = by; p.bz = bz;
    p.projType = 1;
    p.nProjections = n_proj;
    p.globalFactor = global_factor;
    p.epps = epps;
    p.TOF = nbins > 1;
    p.nBins = nbins;
    p.sigma_x = sigma_x;
    p.TOFCenters = tof_centers;
    p.noSensImage = sens == nullptr;
    p.nMeas = 0;
    // corrections (normCoefs[lo], atten image or atten[lo], scatterCoefs[lo])
    p.normalizationCorrection = norm != nullptr;
    p.normCoefs = norm;
    p.attenuationCorrection = atten != nullptr;
    p.CTAttenuation = ct_atten != 0;
    p.atten = atten;
    p.scatterCorrectionMult = scat != nullptr;
    p.scatterCoefs = scat;
    // multi-ray: rays over the crystal pitch (dPitchXY transaxially, dPitchZ axially)
    p.nRays2D = n_rays_xy;
    p.nRays3D = n_rays_z;
    p.dPitchXY = cr_xy;
    p.dPitchZ = cr_z;
    const int64_t n_meas = (int64_t)n_rows * n_cols * n_proj;
    projectorType123Implementation4<T>(p, n_meas, output, xy, z, input, false, false, (uint8_t)(fp ? 1 : 2), sens,
                                       nullptr, n_threads);
    return 0;
}

extern "C" {
/* List-mode events: xyz = 6 coordinates per event (get_detector_coordinates_raw,
 * projector_functions.h:357-368), n_events rays, no TOF. */
int ref_listmode_d(int fp, uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy, double dz, double bx,
                   double by, double bz, int64_t n_events, const double *xyz, double *input, double *output,
                   double *sens, double global_factor, double epps, uint32_t n_threads) {
    paramStruct<double> p;
    p.subsetType = 0;
    p.subsets = 1;
    p.currentSubset = 0;
    p.size_x = 1;
    p.size_y = 1;
    p.dx = dx; p.dy = dy; p.dz = dz;
    p.Nx = nx; p.Ny = ny; p.Nz = nz;
    p.bx = bx; p.by = by; p.bz = bz;
    p.projType = 1;
    p.listMode = 1;
    p.nProjections = 1;
    p.globalFactor = global_factor;
    p.epps = epps;
    p.TOF = false;
    p.nBins = 1;
    double tofc = 0.0;
    p.TOFCenters = &tofc;
    p.noSensImage = sens == nullptr;
    p.nMeas = 0;
    double z0 = 0.0;
    projectorType123Implementation4<double>(p, n_events, output, xyz, &z0, input, false, false, (uint8_t)(fp ? 1 : 2),
                                            sens, nullptr, n_threads);
    return 0;
}
/* Multi-ray sinogram projection: n_rays_xy x n_rays_z rays per LOR. */
int ref_multiray_d(int fp, uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy, double dz, double bx,
                   double by, double bz, uint32_t n_rows, uint32_t n_cols, uint32_t n_proj, const double *xy,
                   const double *z, double *input, double *output, double *sens, uint32_t nbins, double sigma_x,
                   double *tof_centers, double global_factor, double epps, uint32_t n_threads, uint32_t n_rays_xy,
                   uint32_t n_rays_z, double cr_xy, double cr_z) {
    return run<double>(fp, nx, ny, nz, dx, dy, dz, bx, by, bz, n_rows, n_cols, n_proj, xy, z, input, output, sens,
                       nbins, sigma_x, tof_centers, global_factor, epps, n_threads, nullptr, nullptr, 1, nullptr,
                       (uint16_t)n_rays_xy, (uint16_t)n_rays_z, cr_xy, cr_z);
}
/* With PET corrections: norm / scat per measurement of the call (NULL: off);
 * atten: image (ct_atten != 0) or per measurement (ct_atten == 0), NULL: off. */
int ref_siddon_corr_d(int fp, uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy, double dz, double bx,
                      double by, double bz, uint32_t n_rows, uint32_t n_cols, uint32_t n_proj, const double *xy,
                      const double *z, double *input, double *output, double *sens, uint32_t nbins, double sigma_x,
                      double *tof_centers, double global_factor, double epps, uint32_t n_threads, double *norm,
                      double *atten, int ct_atten, double *scat) {
    return run<double>(fp, nx, ny, nz, dx, dy, dz, bx, by, bz, n_rows, n_cols, n_proj, xy, z, input, output, sens,
                       nbins, sigma_x, tof_centers, global_factor, epps, n_threads, norm, atten, ct_atten, scat);
}
/* Projector types 2 / 3 on sinogram data: the voxel-centre arrays are the
 * caller's, padded on both sides with far-away sentinels (the CPU projector
 * reads one past the end of the in-slice centres and, in its first / last
 * slices, rows outside the grid; a sentinel centre is never inside the
 * tube, so those reads end the scan as they would at the grid edge). */
int ref_orth_d(int fp, uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy, double dz, double bx, double by,
               double bz, uint32_t n_rows, uint32_t n_cols, uint32_t n_proj, const double *xy, const double *z,
               double *input, double *output, double *sens, uint32_t nbins, double sigma_x, double *tof_centers,
               double global_factor, double epps, uint32_t n_threads, int proj_type, double orth_width,
               double *x_center, double *y_center, double *z_center, double bmin, double bmax, double vmax,
               double *V, double *norm, double *atten) {
    paramStruct<double> p;
    p.subsetType = 8;
    p.subsets = 1;
    p.currentSubset = 0;
    p.size_x = n_rows;
    p.size_y = n_cols;
    p.dx = dx; p.dy = dy; p.dz = dz;
    p.Nx = nx; p.Ny = ny; p.Nz = nz;
    p.bx = bx; p.by = by; p.bz = bz;
    p.projType = proj_type;
    p.orthWidth = orth_width;
    p.x_center = x_center;
    p.y_center = y_center;
    p.z_center = z_center;
    p.bmin = bmin;
    p.bmax = bmax;
    p.Vmax = vmax;
    p.V = V;
    p.nProjections = n_proj;
    p.globalFactor = global_factor;
    p.epps = epps;
    p.TOF = nbins > 1;
    p.nBins = nbins;
    p.sigma_x = sigma_x;
    p.TOFCenters = tof_centers;
    p.noSensImage = sens == nullptr;
    p.nMeas = 0;
    p.normalizationCorrection = norm != nullptr;
    p.normCoefs = norm;
    p.attenuationCorrection = atten != nullptr;
    p.CTAttenuation = true;
    p.atten = atten;
    const int64_t n_meas = (int64_t)n_rows * n_cols * n_proj;
    projectorType123Implementation4<double>(p, n_meas, output, xy, z, input, false, false, (uint8_t)(fp ? 1 : 2),
                                            sens, nullptr, n_threads);
    return 0;
}
/* The reference's CPU non-local means gradient (NLM.h NLMFunc): interior
 * voxels only (a border of search + patch window is left untouched). */
int ref_nlm_d(double *grad, const double *u_ref, const double *u, const double *gaussian, int32_t sx, int32_t sy,
              int32_t sz, int32_t px, int32_t py, int32_t pz, uint32_t nx, uint32_t ny, uint32_t nz, double h,
              int32_t type, double gamma, double epps, double p, double q, double c, int32_t anatomical) {
    NLMFunc<double>(grad, u_ref, u, gaussian, sx, sy, sz, px, py, pz, nx, ny, nz, (int32_t)(nx * ny), h, type, gamma,
                    epps, p, q, c, anatomical != 0);
    return 0;
}
/* The reference's CPU median filter (MRP.h medianFilter3D) of an image padded
 * by the window on every side (x fastest, padded sizes nx + 2 sx, ...). */
int ref_median_d(const double *padded, double *out, int32_t nx, int32_t ny, int32_t nz, int32_t sx, int32_t sy,
                 int32_t sz) {
    medianFilter3D<double>(padded, out, nx, ny, nz, nx, ny, nz, sx, sy, sz);
    return 0;
}
int ref_siddon_d(int fp, uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy, double dz, double bx, double by,
                 double bz, uint32_t n_rows, uint32_t n_cols, uint32_t n_proj, const double *xy, const double *z,
                 double *input, double *output, double *sens, uint32_t nbins, double sigma_x, double *tof_centers,
                 double global_factor, double epps, uint32_t n_threads) {
    return run<double>(fp, nx, ny, nz, dx, dy, dz, bx, by, bz, n_rows, n_cols, n_proj, xy, z, input, output, sens,
                       nbins, sigma_x, tof_centers, global_factor, epps, n_threads);
}
int ref_siddon_f(int fp, uint32_t nx, uint32_t ny, uint32_t nz, float dx, float dy, float dz, float bx, float by,
                 float bz, uint32_t n_rows, uint32_t n_cols, uint32_t n_proj, const float *xy, const float *z,
                 float *input, float *output, float *sens, uint32_t nbins, float sigma_x, float *tof_centers,
                 float global_factor, float epps, uint32_t n_threads) {
    return run<float>(fp, nx, ny, nz, dx, dy, dz, bx, by, bz, n_rows, n_cols, n_proj, xy, z, input, output, sens,
                      nbins, sigma_x, tof_centers, global_factor, epps, n_threads);
}
}
