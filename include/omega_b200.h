/*
 * omega_b200.h -- C-ABI of the B200 (sm_100a) matrix-free tomographic projectors.
 *
 * This library replaces OMEGA's per-call kernel launch path for the
 * forward projector A*x and the backprojector A^T*y (projector types 1, 4
 * and 5) and the OSEM / PDHG subset updates they drive.  Reference
 * interfaces each entry point replaces are cited beside it (paths inside the
 * OMEGA source tree).
 *
 * Conventions
 *  - Every function returns an int status: OMB_OK (0) or a negative omb_status.
 *    Nothing aborts, traps or exits; the message of the last failure on the
 *    calling thread is returned by omb_last_error().
 *  - Device pointers are plain CUDA device addresses of float32 buffers owned
 *    by the caller (e.g. torch tensors' data_ptr()).  Host pointers are only
 *    read during the call.
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy default
 *    stream.  All work is stream-ordered; nothing synchronises the device
 *    except the functions that return a host scalar (documented below).
 *  - Images are Fortran order (x fastest), length Nx*Ny*Nz.  Measurements are
 *    sinogram/projection order (detector row fastest, then column, then
 *    sinogram/projection in subset order); with TOF the bins are outermost per
 *    call: [bin0 of all rays, bin1 of all rays, ...].
 *  - A handle binds one device (the current device at omb_create) and is not
 *    reentrant: do not call into one handle from two threads at once.
 *    Distinct handles are independent.
 */
#ifndef OMEGA_B200_H
#define OMEGA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OMB_ABI_VERSION 5

typedef enum omb_status {
    OMB_OK = 0,
    OMB_ERR_INVALID = -1,     /* bad argument or geometry */
    OMB_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    OMB_ERR_ALLOC = -3,       /* device allocation failed */
    OMB_ERR_UNSUPPORTED = -4, /* valid request outside what this build implements */
    OMB_ERR_TIMEOUT = -5      /* a bounded device wait gave up */
} omb_status;

typedef enum omb_modality {
    OMB_PET_SINOGRAM = 0, /* PET sinogram: xy = (Ndist*Nang) x [xs, ys, xd, yd]; z = nProj x [zs, zd] */
    OMB_CT_PANEL = 1,     /* CT flat panel: xy = nProj x [sx, sy, sz, dx, dy, dz]; z = nProj x [ux*pitchX, uy*pitchX] */
    OMB_PET_LISTMODE = 2, /* PET list-mode events (getDetectorCoordinatesListmode, general_opencl_functions.h:
                             1304-1320): xy = events x [xs, ys, zs, xd, yd, zd] in subset order, z unused (n_z 0
                             allowed); n_proj = events, n_rows_d = n_cols_d = 1, n_meas = cumulative events */
    OMB_PET_INDEXED = 3   /* PET index-based events (general_opencl_functions.h:1277-1301): xy = crystal table
                             [x, y] per transaxial detector, z = axial positions; per event the detector index
                             pairs tr_index[2e..2e+1] and ax_index[2e..2e+1]; sizes as OMB_PET_LISTMODE */
} omb_modality;

typedef enum omb_read_precision {
    OMB_READ_FP32 = 0, /* forward projections read the FP32 image (default) */
    OMB_READ_BF16 = 1  /* forward projections read a BF16 rounding of it; accumulation stays FP32 */
} omb_read_precision;

typedef enum omb_bp_mode {
    OMB_BP_FLOAT_ATOMIC = 0, /* float32 atomics (the reference's CUDA path); projector type 5: the reference's
                                voxel-driven gather (projectorType5Backward) */
    OMB_BP_FIXED64 = 1,      /* int64 fixed point, bit-identical run to run (the reference's OpenCL -DATOMIC path);
                                projector type 5: the ray-driven scatter below with int64 atomics */
    OMB_BP_RAY = 2           /* projector type 5: the ray-driven scatter form, the exact adjoint of the forward
                                projection (projectorType5Forward), float atomics; other types: as
                                OMB_BP_FLOAT_ATOMIC (their backprojections are ray-driven already) */
} omb_bp_mode;

/*
 * Geometry and projector options.  Mirrors the scalars and arrays OMEGA's
 * Python layer uploads before the first launch
 * (omegatomo/projector/init.py:468-703, kernel-argument prefixes kIndF/kIndB)
 * in an explicit, versioned layout: `struct_size` must equal
 * sizeof(omb_geometry_desc) and `abi_version` OMB_ABI_VERSION.
 * All arrays are host pointers, copied to the device by omb_create.
 */
typedef struct omb_geometry_desc {
    uint32_t struct_size;
    uint32_t abi_version;
    int32_t modality;        /* omb_modality */
    int32_t fp_type;         /* forward projector: 1 (improved Siddon), 2 (orthogonal distance), 3 (volume of
                                intersection), 4 (interpolation), 5 (branchless distance-driven) */
    int32_t bp_type;         /* backprojector: 1 to 5 */
    uint32_t nx, ny, nz;     /* image size */
    float dx, dy, dz;        /* voxel size (mm) */
    float bx, by, bz;        /* FOV corner (mm), the lower edge of voxel 0 */
    uint32_t n_rows_d;       /* Ndist (PET) / detector rows (CT) */
    uint32_t n_cols_d;       /* Nang (PET) / detector columns (CT) */
    int64_t n_proj;          /* sinograms / projections in total */
    int32_t n_subsets;
    int32_t subset_type;     /* OMEGA subsetType: 8-11 whole sinograms/projections; 1, 2, 4, 5 measurement-level (PET) */
    const int64_t *n_meas;   /* n_subsets+1 cumulative sinogram/projection counts (proj.py nMeas) */
    const float *xy;         /* see omb_modality; CT rows in subset order */
    int64_t n_xy;            /* number of floats in xy */
    const float *z;          /* see omb_modality; in subset order for subset types >= 8 */
    int64_t n_z;             /* number of floats in z */
    float dpitch_x, dpitch_y;/* detector pitch (proj.py dPitchX/dPitchY) */
    float global_factor;     /* proj.py global_factor */
    float epps;              /* proj.py epps */
    int32_t tof_bins;        /* 1 = no TOF */
    float sigma_x;           /* TOF Gaussian sigma (mm) */
    const float *tof_centers;/* tof_bins centres (mm) (proj.py TOFCenter) */
    float dL;                /* type 4 step length (mm), coordinates.py:242-262 */
    float d_scale4[3];       /* type 4 1/(d*N) per axis */
    float d_size5[2];        /* type 5 dSizeX, dSizeY */
    float d_scale5[3];       /* type 5 dScaleX/Y/Z */
    float kerroin;           /* type 4 CT backprojection weight */
    int32_t fixed64_workspace; /* nonzero: allocate the int64 accumulators omb_backward needs for OMB_BP_FIXED64 */
    const uint16_t *tr_index;  /* OMB_PET_INDEXED: 2 x n_proj transaxial detector indices (source, detector) */
    const uint16_t *ax_index;  /* OMB_PET_INDEXED: 2 x n_proj axial indices into z */
    int32_t n_rays_xy;         /* PET multi-ray (proj.py n_rays_transaxial, 0 or 1: one ray): rays per LOR
                                  spread over dpitch_x transaxially */
    int32_t n_rays_z;          /* (n_rays_axial) rays spread over dpitch_y axially; projector type 1 only */
    /* Projector types 2 / 3 (PET; the tube of response of projectorType123.cl -DORTH / -DVOL).  The image must
     * be square transaxially (nx == ny, dx == dy, bx == by). */
    float tube_width;          /* type 2: options.tube_width_z (mm), the distance where the weight reaches 0 */
    float tube_radius;         /* type 3: options.tube_radius (mm) */
    int32_t orth_xy;           /* options.orthTransaxial: the tube spreads in the slice (CRYSTXY) */
    int32_t orth_z;            /* options.orthAxial: the tube spreads axially (CRYSTZ) */
    float vol_bmin, vol_bmax, vol_vmax; /* type 3: options.bmin, bmax, Vmax (coordinates.py:192-206) */
    const float *vol_v;        /* type 3: options.V, the intersection volume per 1/1000 mm above bmin */
    int64_t n_vol_v;           /* entries in vol_v */
} omb_geometry_desc;

typedef struct omb_handle omb_handle;

/* Library ABI version (OMB_ABI_VERSION of the build). */
int omb_abi_version(void);

/* Message of the last failure on the calling thread ("" if none). Valid until the next call on this thread. */
const char *omb_last_error(void);

/*
 * Validate the geometry, upload it to the current device and return a handle.
 * Replaces omegatomo/projector/init.py:39-703 (initProjector: option
 * assembly, device uploads, kernel JIT) and ProjectorClass.h:1780
 * (addProjector) / 3055 (createBuffers) / 3117 (initializeKernel).
 */
int omb_create(const omb_geometry_desc *desc, omb_handle **out);

/* Free all device memory of the handle. Replaces nothing: OMEGA frees on garbage collection. */
int omb_destroy(omb_handle *h);

/* Measurement count of one subset (all TOF bins), or of all subsets when subset == -1. */
int64_t omb_measurement_count(const omb_handle *h, int32_t subset);

/* Image voxel count Nx*Ny*Nz. */
int64_t omb_image_count(const omb_handle *h);

/*
 * y = A_s * image.  subset in [0, n_subsets) or -1 for all subsets in one
 * launch (output concatenated in subset order).  `y` is overwritten.
 * Replaces omegatomo/projector/projfunctions.py:86-436 (forwardProjection,
 * CuPy branch) and ProjectorClass.h:3478 (forwardProjection); kernels
 * restate projectorType123.cl:81-1374 (-DFP -DSIDDON), projectorType4.cl:84
 * (projectorType4Forward) and projectorType5.cl:64 (projectorType5Forward).
 */
int omb_forward(omb_handle *h, int32_t subset, const float *image, float *y, void *stream);

/*
 * Forward projection of n_frames images in one launch (frames of a dynamic
 * study share the geometry): y[f*y_stride ...] = A_s images[f*image_stride ...].
 * Each ray is traced once for up to eight frames.  TOF handles take
 * n_frames == 1.  Replaces the per-timestep FP launches of the reference's
 * loop (reconstructionAF.h:1089-1190, one launch per frame).
 */
int omb_forward_frames(omb_handle *h, int32_t subset, int32_t n_frames, const float *images, int64_t image_stride,
                       float *y, int64_t y_stride, void *stream);

/*
 * image = A_s^T * y, and sens = A_s^T * 1 when `sens` is not NULL (the
 * reference's no_norm == 0 pass).  Both outputs are overwritten.
 * mode: omb_bp_mode; OMB_BP_FIXED64 needs a handle created with
 * fixed64_workspace != 0.  Projector type 5 has two backprojectors: the
 * voxel-driven gather of the reference (OMB_BP_FLOAT_ATOMIC; not the exact
 * adjoint of the forward projection) and the ray-driven scatter
 * (OMB_BP_RAY, or OMB_BP_FIXED64 for its deterministic int64 form), which
 * is.
 * Replaces projfunctions.py:735-1095 (backwardProjection) and
 * ProjectorClass.h:3893 (backwardProjection); kernels restate
 * projectorType123.cl (-DBP, rhs() general_opencl_functions.h:1212-1275),
 * projectorType4.cl:718 (projectorType4Backward) and projectorType5.cl:381.
 */
int omb_backward(omb_handle *h, int32_t subset, const float *y, float *image, float *sens,
                 int32_t mode, void *stream);

/*
 * Backprojection of n_frames measurement vectors into n_frames images (float
 * atomics; images overwritten).  Replaces the per-timestep BP launches of
 * reconstructionAF.h:1265.
 */
int omb_backward_frames(omb_handle *h, int32_t subset, int32_t n_frames, const float *y, int64_t y_stride,
                        float *images, int64_t image_stride, void *stream);

/*
 * One OSEM sub-iteration for PET, fused on the device:
 *   fp = A_s x + epps;  r = y_s / fp (NaN/Inf -> epps);  rhs = A_s^T r;
 *   x = x / sens_s * (rhs + epps)
 * `sens` is the subset's sensitivity image already clamped to >= epps
 * (see omb_sensitivity).  `work_meas` is caller scratch of
 * omb_measurement_count(h, subset) floats; `work_img` of Nx*Ny*Nz floats.
 * Restates computeForwardProject.h:20-21, 92-95, 400-401 (ratio),
 * algorithms.h:12-15 with subiterStep.h:110-121 (EM update).
 */
int omb_osem_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset,
                    const float *sens, float *work_meas, float *work_img, void *stream);

/*
 * sens = max(A_s^T 1, epps): the per-subset sensitivity image of the first
 * iteration (reconstructionAF.h:303-328 with the clamp of functions.hpp:2980-2996).
 */
int omb_sensitivity(omb_handle *h, int32_t subset, float *sens, void *stream);

/*
 * One OSEM sub-iteration for a batch of n_frames images that share the
 * geometry and the subset's sensitivity image `sens` (omb_sensitivity):
 * for every frame f, fp = A_s x_f, r = y_f / (fp + epps) (NaN/Inf -> epps),
 * x_f = x_f / sens * (A_s^T r + epps) -- the reference's per-timestep OSEM
 * step (reconstructionAF.h:1089-1265 with computeForwardProject.h:4-101 and
 * algorithms.h:12-15) for all frames with one forward and one backward
 * launch (type 1 shares each ray walk between frames).  images: frame f at
 * images + f * image_stride; y_subset: this subset's measurements of frame f
 * at y_subset + f * y_stride; work_meas holds n_frames *
 * omb_measurement_count(h, subset) floats, work_img n_frames * Nx*Ny*Nz.
 * Projector types 1 and 4, PET.
 */
int omb_osem_subset_frames(omb_handle *h, int32_t subset, int32_t n_frames, float *images, int64_t image_stride,
                           const float *y_subset, int64_t y_stride, const float *sens, float *work_meas,
                           float *work_img, void *stream);

/*
 * Total voxel intersections (sum over the subset's rays of the Siddon walk
 * length Np) written to *out_host; synchronises `stream`.  The
 * algorithmic-byte model of the projector roofline counts bytes per
 * intersection.  The reference has no counterpart (its pre-loop computes Np
 * per ray inside the kernel, general_opencl_functions.h:1873, 1942).
 */
int omb_intersection_count(omb_handle *h, int32_t subset, int64_t *out_host, void *stream);

/*
 * Number of weights the handle's resident system matrix holds for `subset`
 * (omb_tuning.siddon_bp_matrix; built by the subset's first projection
 * through it), 0 when none is built.  Host only; no counterpart in the
 * reference (its projectors hold no matrix).
 */
int omb_system_matrix_nnz(omb_handle *h, int32_t subset, int64_t *out_host);

/*
 * Launch shapes of a handle's projector kernels.  omb_create sets the
 * defaults below; omb_autotune times the candidates on the handle's own
 * geometry and keeps the fastest; omb_set_tuning sets them directly.  The
 * shapes change only how the work is split, not what is computed: results
 * agree to FP32 rounding (the order of additions differs).  No counterpart in
 * the reference, whose kernels have fixed launch shapes.
 */
typedef struct omb_tuning {
    uint32_t struct_size;            /* sizeof(omb_tuning) */
    int32_t siddon_blocks_per_sm;    /* 1..32 (default 8): grid of the grid-stride Siddon kernels */
    int32_t siddon_frames_per_walk;  /* 1, 2, 4, 8 (default 8): most frames sharing one ray walk */
    int32_t bdd_fp_columns;          /* 8, 16 (default 8): type-5 forward, detector columns per thread */
    int32_t bdd_bp_zrun;             /* 4, 8, 16 (default 8): type-5 backward, voxels along z per thread */
    int32_t bdd_fp_block_rows;       /* 4, 8 (default 8): type-5 forward, warps per block */
    int32_t bdd_bp_block_rows;       /* 4, 8 (default 8): type-5 backward, warps per block */
    int32_t siddon_frame_layout;     /* 0, 1 (default 1): type-1 non-TOF batches of >= 4 frames.
                                        0: the kernels read and update each frame's image in place;
                                        1: through a voxel-interleaved copy (the 4 or 8 frames of a walk
                                        stored together per voxel: 16-byte loads, float4 atomics), kept
                                        on the handle (ceil(frames / 8) * 8 images, allocated by the
                                        first such call made outside CUDA-graph capture; calls on one
                                        handle must therefore be ordered on one stream) */
    int32_t siddon_fp_steps;         /* 1, 2, 4 (default 4): non-TOF type-1 forward walks compute this
                                        many crossings before gathering their voxels, so that many
                                        loads are in flight per thread */
    int32_t bdd_fp_staged;           /* 0, 1 (default 1): type-5 forward projection with each CTA's
                                        per-slice image boxes staged in shared memory by TMA (applies
                                        with bdd_fp_columns = 8; needs Nx, Ny multiples of 4) */
    int32_t bdd_bp_staged;           /* 0, 1 (default 1): type-5 backprojection with each CTA's
                                        per-projection detector boxes staged in shared memory by TMA
                                        (applies with bdd_bp_zrun = 8 or 16; needs a row count that is a
                                        multiple of 4) */
    int32_t siddon_bp_matrix;        /* 0, 1 (default 0): type-1, 2 and 3 non-TOF backprojections of
                                        measurements through a transposed system matrix kept on the handle
                                        (the Siddon or tube weights; types 2 / 3 also project forward
                                        through a ray-major copy when fp_type == bp_type, and fall back to
                                        the tracers when it does not fit in memory) (per subset:
                                        for every voxel the weights of the rays crossing it, 8 bytes a
                                        crossing), built by the first such call on a subset (that call
                                        synchronises its stream and must not be captured into a CUDA
                                        graph); one thread per voxel, no atomics, the sums in ray order:
                                        bit-identical call to call.  Sensitivity images keep the
                                        ray-driven kernels */
} omb_tuning;

/*
 * Image read precision of the forward projections of types 1 and 4
 * (omb_read_precision).  With OMB_READ_BF16 every forward call first rounds
 * its images to BF16 (round to nearest even) into copies owned by the handle
 * and the kernels read those: half the image bytes per sample, FP32
 * accumulation; the relative L2 error against the FP64 oracle is stated per
 * projector by the tests (below 4e-3).  max_frames: the most images one
 * forward call may carry; the copies are allocated here, not during a
 * forward call.  No counterpart in the reference (its images are FP32
 * textures).
 */
int omb_set_read_precision(omb_handle *h, int32_t mode, int32_t max_frames);

int omb_get_tuning(const omb_handle *h, omb_tuning *out);

/*
 * The built-in reconstruction behind one call (the reference's compiled
 * omegaMain entry, libHeader.h:1466, with reconstructionAF.h:1053-1500, for
 * the algorithms of this path).  Explicit parameters instead of the
 * reference's 200-field options struct.
 */
typedef enum omb_recon_algorithm {
    OMB_RECON_OSEM = 1,     /* options.OSEM: per-subset sensitivity images, EM update per subset (PET) */
    OMB_RECON_PDHG_TV = 2,  /* options.PDHG with options.TV: one subset, smoothed TV gradient */
    OMB_RECON_OSL_OSEM = 3, /* options.OSL_OSEM: one-step-late OSEM, x / (sens + dU) * rhs, dU = beta * the
                               prior's gradient at the current image (priors.h:376-451) */
    OMB_RECON_ROSEM = 4,    /* options.ROSEM: x + lam * x / sens * (rhs - sens) per subset (algorithms.h:102-106) */
    OMB_RECON_RAMLA = 5,    /* options.RAMLA: x + lam * rhs * x with rhs the backprojection of y / fp - 1
                               (computeForwardProject.h:98-122, auxKernels.cl:1997-2026) */
    OMB_RECON_BSREM = 6,    /* options.BSREM: RAMLA sub-iterations, then once per iteration the MAP step
                               x -= lam * x * dU, x >= epps (iterStep.h:14-34, algorithms.h:130-135) */
    OMB_RECON_ROSEM_MAP = 7,/* options.ROSEM_MAP: ROSEM sub-iterations, then the same MAP step */
    OMB_RECON_PKMA = 8,     /* options.PKMA: x_a = max(epps, x - lam * (A^T (1 - y / fp) + dU)), x = (1 - a) x +
                               a x_a per subset (algorithms.h:151-212, auxKernels.cl:2008-2018); dU only with a prior */
    OMB_RECON_MRAMLA = 9,   /* options.MRAMLA: x = x + lam * A^T (y / fp - 1), clamped to [epps, U) (algorithms.h:31-52) */
    OMB_RECON_MBSREM = 10   /* options.MBSREM: the same with dU added to the backprojection (priors.h:361-370) */
} omb_recon_algorithm;

typedef enum omb_prior {
    OMB_PRIOR_RDP = 1,      /* options.RDP: relative difference prior, parameter rdp_gamma */
    OMB_PRIOR_QUAD = 2,     /* options.Quad: the quadratic window (prior_window) applied with mirrored edges */
    OMB_PRIOR_HUBER = 3,    /* options.Huber: the same with the gradient clamped to +-huber_delta */
    OMB_PRIOR_NLM = 4,      /* options.NLM (with NLTV / NLM_MRP / NLRD / NLLange / NLGGMRF): omb_nlm_gradient */
    OMB_PRIOR_MRP = 5,      /* options.MRP: omb_mrp_gradient over the prior_g window (Ndx, Ndy, Ndz) */
    OMB_PRIOR_TV = 6,       /* options.TV with a MAP algorithm other than PDHG: omb_tv_gradient, tv_smoothing */
    OMB_PRIOR_GGMRF = 7,    /* options.GGMRF: omb_ggmrf_gradient over prior_g with ggmrf_weights and ggmrf[3] */
    OMB_PRIOR_HYPERBOLIC = 8,/* options.hyperbolic: omb_hyperbolic_gradient over prior_g with hyper_weights */
    OMB_PRIOR_WMEAN = 9,    /* options.weighted_mean, mean_type 1-6: omb_wmean_gradient over prior_g */
    OMB_PRIOR_AD = 10,      /* options.AD: omb_ad_gradient with ad_dt, ad_k, ad_niter, ad_flux, ad_diffusion */
    OMB_PRIOR_LFILTER = 11, /* options.L: omb_lfilter_gradient over prior_g with lfilter_weights */
    OMB_PRIOR_FMH = 12      /* options.FMH: omb_fmh_gradient over prior_g with fmh_weights */
} omb_prior;

typedef struct omb_recon_params {
    uint32_t struct_size;     /* sizeof(omb_recon_params) */
    int32_t algorithm;        /* omb_recon_algorithm */
    int32_t n_iter;           /* options.Niter */
    float beta;               /* PDHG: TV weight (options.beta) */
    float tv_smoothing;       /* PDHG: options.TVsmoothing */
    float tau;                /* PDHG primal step (options.tauCP); <= 0: 1 / the power-method eigenvalue */
    float sigma;              /* PDHG dual step (options.sigmaCP) */
    float theta;              /* PDHG extrapolation (options.thetaCP) */
    int32_t power_iterations; /* options.powerIterations (0: 20) */
    int32_t positivity;       /* options.enforcePositivity */
    int32_t use_graph;        /* nonzero: capture one iteration as a CUDA graph and replay it */
    float tau_used;           /* out: the primal step of the run */
    float rdp_gamma;          /* OSL-OSEM, BSREM, ROSEM-MAP: options.RDP_gamma (beta is options.beta) */
    int32_t prior;            /* OSL-OSEM, BSREM, ROSEM-MAP: omb_prior */
    const float *prior_window;/* Quad / Huber: device window of (2g0+1)(2g1+1)(2g2+1) weights, x fastest: the
                                 neighbours' -w and the centre sum(w) (libHeader.h:1147-1154) */
    int32_t prior_g[3];       /* Quad / Huber: options.Ndx, Ndy, Ndz */
    float huber_delta;        /* Huber: options.huber_delta */
    const float *relaxation;  /* ROSEM / RAMLA / BSREM / ROSEM-MAP / PKMA / MRAMLA / MBSREM: host, n_iter values
                                 lam[iter] (options.lambdaN); NULL: 1 / (iter / 20 + 1) (prepass.py:962-972) */
    const float *momentum;    /* PKMA: host, n_iter * n_subsets values alpha[iter * n_subsets + subset]
                                 (options.alpha_PKMA); NULL: 1 + 0.45 k / (k + 100), k the sub-iteration count
                                 (prepass.py:998-1006) */
    float upper_bound;        /* MRAMLA / MBSREM: options.U; <= 0: 10000 (prepass.py:955-959) */
    int32_t nlm_type;         /* OMB_PRIOR_NLM: 0 NLM, 1 NLTV, 2 NLM-MRP, 3 NLRD, 4 NL Lange, 5 MRP + Lange, 6 NLGGMRF;
                                 the search window is prior_g (Ndx, Ndy, Ndz), gamma is rdp_gamma */
    int32_t nlm_patch[3];     /* options.Nlx, Nly, Nlz */
    float nlm_h;              /* options.NLMsigma^2 (libHeader.h:1285-1286) */
    const float *nlm_gaussian;/* device: (2 Nlx + 1)(2 Nly + 1)(2 Nlz + 1) patch weights, x fastest */
    const float *nlm_ref;     /* device reference image of the patch distances (NLM_use_anatomical), or NULL */
    float ggmrf[3];           /* NLGGMRF: options.GGMRF_p, GGMRF_q, GGMRF_c */
    int32_t nlm_adaptive;     /* options.NLAdaptive */
    float nlm_adaptive_s;     /* options.NLAdaptiveConstant */
    int32_t precond;          /* PKMA / MRAMLA / MBSREM image preconditioner: 0 none, 1 type 0 (rhs / D), 2 type 1
                                 (rhs * x / D), 3 type 2 (rhs * max(x, max(1e-5, precond_ref)) / D), see
                                 omb_precond_image */
    int32_t mrp_no_norm;      /* MRP: options.med_no_norm */
    const float *ggmrf_weights;/* GGMRF: device, the neighbours' weights (centre left out, z fastest) */
    const float *hyper_weights;/* hyperbolic: device, options.weights_quad (centre left out, x fastest) */
    float hyper_delta;        /* hyperbolic: options.hyperbolicDelta */
    const float *wmean_weights;/* weighted mean: device, options.weighted_weights (x fastest) */
    int32_t wmean_type;       /* weighted mean: options.mean_type (1-3 arithmetic, harmonic, geometric; 4-6 their
                                 neighbourhood forms, see omb_wmean_gradient); the
                                 normalisation switch is mrp_no_norm (options.med_no_norm) */
    int32_t tv_variant;       /* OMB_PRIOR_TV and PDHG: omb_tv_variant (0: the plain TV) */
    float tv_sigma;           /* OMB_PRIOR_TV and PDHG: options.SATVPhi (SATV, weighted TV) */
    float tv_c;               /* OMB_PRIOR_TV and PDHG: options.C (anatomical type 2) or options.eta (type 5,
                                 APLS) */
    const float *tv_ref;      /* OMB_PRIOR_TV and PDHG: device reference image / tensor of the anatomical
                                 variants (OMB_TV_ANAT1 and above), NULL otherwise */
    float wmean_wsum;         /* weighted mean: the sum of wmean_weights (the means divide the weights by it;
                                 types 4-6 also weight their sum by the raw weights); <= 0: 1 */
    int32_t tv_prox;          /* PDHG: nonzero = proximal TV (options.ProxTV: a dual TV variable projected onto
                                 the beta ball, omb_proxtv_dual / omb_proxtv_divergence) instead of the TV
                                 gradient */
    float sigma2;             /* PDHG with proximal TV: the TV dual step (options.sigma2CP) */
    int32_t l2_ball;          /* PDHG with proximal TV: options.useL2Ball (1: L2 ball, 0: max-norm ball) */
    int32_t diff_type;        /* options.derivativeType: PDHG with proximal TV (0 forward, 1 backward
                                 differences) and the gradient image preconditioner (0, 1, or 2 central) */
    const float *precond_ref; /* PKMA / MRAMLA / MBSREM, precond = 3 (options.precondTypeImage[2]): device
                                 reference image (options.referenceImage) */
    const float *precond_alpha;/* PKMA / MRAMLA / MBSREM, options.precondTypeImage[3]: host, n_iter * n_subsets
                                 values (options.alphaPrecond) the gradient is multiplied by, or NULL */
    int32_t precond_grad;     /* options.precondTypeImage[4]: gradient-based preconditioner (functions.hpp:
                                 2036-2054), recomputed in sub-iterations grad_iters[0] .. grad_iters[1] and
                                 applied from grad_iters[0] on */
    float grad_v[2];          /* options.gradV1, gradV2: its bounds */
    int32_t grad_iters[2];    /* options.gradInitIter, gradLastIter (sub-iteration counts) */
    int32_t precond_curv;     /* options.precondTypeImage[6]: curvature preconditioner dP = sum over the
                                 subsets of S / A_s^T (A_s 1 / y_s) (reconstructionAF.h:600-650) */
    int32_t precond_meas;     /* options.precondTypeMeas[0]: the ratio divided by A_s 1 (zeros -> 1) */
    int32_t pkma_relax;       /* PKMA: bit 0 options.computeRelaxationParameters (lam from the norms of the
                                 image and the gradient, algorithms.h:155-187), bit 1 options.relaxationScaling */
    const float *filter_h;    /* PDHG, options.precondTypeMeas[1]: device, filter_nf taps h = ifft(filter) of the
                                 filtering-based measurement preconditioner (see omb_row_filter), or NULL */
    const float *filter_hinv; /* the taps of 1 / (1 + sigma filter) (the dual step's inverse filter; needed when
                                 filter_iters > 0) */
    int32_t filter_nf;        /* the filters' length Nf (a power of two >= filter_rows) */
    int32_t filter_rows;      /* detector rows per filtered column (nRowsD) */
    int32_t filter_iters;     /* options.filteringIterations: the iterations that filter (0: all, with the plain
                                 dual step) */
    float tau_filt;           /* options.tauCPFilt: the primal step while filtering; <= 0: 1 / the power-method
                                 eigenvalue of A^T F A */
    int32_t tgv;              /* PDHG: options.TGV, the proximal TGV (omb_proxtgv_step) in place of the TV term:
                                 0 off, 1 3-D (TGVZ), 2 2-D (options.use2DTGV); the dual step divides by
                                 1 + sigma beta (computeForwardProject.h:295-298) and the filter by sigma beta */
    float alpha0_tgv;         /* options.alpha0TGV: the first-order ball (q) */
    float alpha1_tgv;         /* options.alpha1TGV: the second-order ball (r) */
    const float *img_filter_h;/* options.precondTypeImage[5] (PKMA / MRAMLA / MBSREM, PDHG): device, the 1-D taps
                                 of the filtering-based image preconditioner (see omb_image_filter), or NULL;
                                 applied last in the image preconditioning of sub-iterations k < filter_iters
                                 (filter_iters 0: k = 0 only); PDHG switches its step to tau (the power method
                                 without the filter) at k = filter_iters */
    int32_t img_filter_nf;    /* its length Nf (a power of two >= nx, ny) */
    float tau_used2;          /* out: PDHG with a filtering preconditioner, the primal step from iteration
                                 filter_iters on (0 when the run never switches) */
    float ad_dt;              /* OMB_PRIOR_AD: options.TimeStepAD */
    float ad_k;               /* OMB_PRIOR_AD: options.KAD (conductance) */
    int32_t ad_niter;         /* OMB_PRIOR_AD: options.NiterAD */
    int32_t ad_flux;          /* OMB_PRIOR_AD: options.FluxType (1 exponential, 2 quadratic) */
    int32_t ad_diffusion;     /* OMB_PRIOR_AD: options.DiffusionType (1 gradient, 2 modified curvature); the
                                 normalisation switch is mrp_no_norm (options.med_no_norm) */
    int32_t rdp_edge;         /* OMB_PRIOR_RDP: 1 neighbours outside the image clamped to the edge voxel (options.useImages,
                                 the reference's default), 0 read as 0 (see omb_rdp_gradient_ex) */
    const float *lfilter_weights;/* OMB_PRIOR_LFILTER: device, options.a_L (one weight per rank of the window) */
    const float *fmh_weights; /* OMB_PRIOR_FMH: device, options.fmh_weights ((2 Ndx + 1) x lines, column-major) */
} omb_recon_params;

/*
 * Runs p->n_iter iterations from x0 (device, one image) into x_out (device).
 * y (device): OSEM, the measurements of all subsets concatenated in subset
 * order, each subset as omb_osem_subset takes it (TOF bins outermost); PDHG,
 * the measurement vector of all subsets (omb_measurement_count(h, -1)).
 * Allocates its scratch with cudaMallocAsync on `stream` (OSEM: one image
 * per subset for the sensitivities) and synchronises `stream` on return.
 */
int omb_reconstruct(omb_handle *h, omb_recon_params *p, const float *y, const float *x0, float *x_out, void *stream);

/*
 * One one-step-late OSEM sub-iteration (subiterStep.h:219-226): as
 * omb_osem_subset, with the update image / (sens + du) * rhs; du (device,
 * one image) is the prior gradient including its weight.
 */
int omb_osl_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const float *sens,
                   const float *du, float *work_meas, float *work_img, void *stream);

typedef enum omb_tv_variant {
    OMB_TV_PLAIN = 0,  /* TVtype 1-3 without a reference image: the plain smoothed TV */
    OMB_TV_SATV = 1,   /* TVtype 4 (SATV), sigma = options.SATVPhi */
    OMB_TV_W1 = 2,     /* TVtype 6 (weighted TV, TVW1), sigma = options.SATVPhi */
    OMB_TV_ANAT1 = 3,  /* TV_use_anatomical, TVtype 1: ref = the 9-channel tensor (9 images, channel 3 r + c) */
    OMB_TV_ANAT2 = 4,  /* TV_use_anatomical, TVtype 2: ref = the reference image, C = options.C */
    OMB_TV_APLS = 5    /* TV_use_anatomical TVtype 5, and APLS: ref = the reference image, C = options.eta */
} omb_tv_variant;

/*
 * Smoothed TV gradient (priors.h:404-409, TVKernel auxKernels.cl:1733-1990,
 * plain TV; neighbours outside the image read the edge voxel): grad += beta *
 * grad TV(u) with the smoothing `smooth` (options.TVsmoothing).
 */
int omb_tv_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float beta, float smooth,
                    void *stream);

/*
 * Detector-row filter of the filtering-based measurement preconditioner
 * (applyMeasPreconditioning functions.hpp:2109-2166, filtering :1882-1902):
 * every column of n_rows values (rows fastest; n_cols columns) zero-padded
 * to nf, filtered by a real even filter in the Fourier domain and cut back:
 * out[i] = sum_j h[(i - j) mod nf] in[j], h = ifft(filter) (device, nf
 * taps).  in and out (device) must differ; n_rows <= 2048, nf >= n_rows.
 */
int omb_row_filter(const float *in, float *out, int32_t n_rows, int64_t n_cols, const float *h, int32_t nf,
                   void *stream);

/*
 * The filtering-based image preconditioner (filtering2D functions.hpp:
 * 1908-1932, applied by applyImagePreconditioning :2093-2099): every slice of
 * g (device, nx x ny x nz, x fastest) zero-padded to nf x nf, multiplied in the
 * Fourier domain by the separable filter F = f f^T / max(f f^T) and cut back
 * to nx x ny; computed as the circular convolution of the x lines, then the y
 * lines, with h = real(ifft(f)) / sqrt(max(f f^T)) (device, nf taps).  tmp
 * (device, one image) is scratch; g is filtered in place.  nx, ny <= nf <= 2048.
 */
int omb_image_filter(float *g, float *tmp, int32_t nx, int32_t ny, int32_t nz, const float *h, int32_t nf,
                     void *stream);

/*
 * Proximal TV of the PDHG loop (priors.h:261-281; ProxTVGradient, ProxTVq,
 * ProxTVDivergence auxKernels.cl:1141-1343).  q (device) holds 3 images
 * (x, y, z components, x fastest), zero before the first iteration.
 *   omb_proxtv_dual:       q <- P(q + sigma2 D x), D the forward differences
 *                          (diff_type 0; -x at the last voxel) or backward
 *                          ones (1; x at the first), P the projection onto the
 *                          per-voxel ball of radius alpha (options.beta):
 *                          L2 (l2_ball != 0) or max norm;
 *   omb_proxtv_divergence: rhs -= div q (backward differences for
 *                          diff_type 0, forward for 1), before the primal step.
 */
int omb_proxtv_dual(const float *x, float *q, int32_t nx, int32_t ny, int32_t nz, float sigma2, float alpha,
                    int32_t l2_ball, int32_t diff_type, void *stream);
int omb_proxtv_divergence(const float *q, float *rhs, int32_t nx, int32_t ny, int32_t nz, int32_t diff_type,
                          void *stream);

/*
 * One proximal TGV step of the PDHG loop (priors.h:284-313; ProxTVGradient
 * with PROXTGV, ProxTVq, ProxTVDivergence, ProxTGVSymmDeriv, ProxTGVq,
 * ProxTGVDivergence auxKernels.cl:1141-1560; forward differences, the only
 * form the reference's kernels build):
 *   q <- P_alpha0(q + sigma2 (D x - v)),   rhs -= div q,
 *   r <- P_alpha1(r + sigma2 E v),         E v the symmetric derivative,
 *   v1 = v + tau (q + div_sym r),          v <- v1 + theta (v1 - v).
 * three_d != 0: v holds 3 images, r 6 (rxx, ryy, rzz, rxy, rxz, ryz);
 * three_d == 0 (use2DTGV): v 2 images, r 3 (rxx, ryy, rxy), and the z
 * difference of x enters q without a v term.  q holds 3 images.  All
 * device, x fastest, zero before the first iteration.  The balls are
 * per-voxel L2 (off-diagonal terms of r counted twice; l2_ball != 0) or
 * max-norm.
 */
int omb_proxtgv_step(const float *x, float *q, float *r, float *v, float *rhs, int32_t nx, int32_t ny, int32_t nz,
                     float sigma2, float alpha0, float alpha1, float theta, float tau, int32_t l2_ball, int32_t three_d,
                     void *stream);

/*
 * The TV gradients of the other TV settings (TVKernel built with -DSATV,
 * -DTVW1, -DANATOMICAL1/2/3; ProjectorClass.h:900-918, functions.hpp:
 * 1096-1113): grad += beta * dTV_variant(u), smoothing `smooth`
 * (TVsmoothing, APLSsmoothing for APLS); `ref` (device) the reference image
 * or tensor of the anatomical variants, NULL otherwise.  OMB_TV_PLAIN is
 * omb_tv_gradient.
 */
int omb_tv_gradient_ex(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float beta, float smooth,
                       int32_t variant, float sigma, float C, const float *ref, void *stream);

/*
 * GGMRF prior gradient (GGMRFKernel, auxKernels.cl:878-980; the image read
 * clamped to its edges): grad += beta * sum_k w_k |d|^(p-1) / (1 + |d/c|^(p-q))
 * (p - pqc |d|^(p-q) / (1 + |d/c|^(p-q))) sign(d), d = u_j - u_k, over the
 * (2sx+1)(2sy+1)(2sz+1) - 1 neighbours in the order x outermost, z fastest,
 * pqc = (p - q) / c^(p-q); `weights` device (quadWeights of the GGMRF branch).
 */
int omb_ggmrf_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t sx, int32_t sy,
                       int32_t sz, const float *weights, float p, float q, float c, float beta, void *stream);

/*
 * Hyperbolic prior gradient (hyperbolicKernel, auxKernels.cl:1591-1688; the
 * image read clamped to its edges): grad += beta * sum_k w_k t / delta /
 * sqrt(t^2 + 1), t = (u_j - u_k) / delta, neighbours z outermost, x fastest,
 * `weights` (device) the quadratic prior's normalised weights.
 */
int omb_hyperbolic_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t sx, int32_t sy,
                            int32_t sz, const float *weights, float delta, float beta, void *stream);

/*
 * Weighted-mean prior gradient (priors.h:99-210).  Types 1-3: m = the
 * weighted arithmetic / harmonic / geometric mean of the mirrored
 * (2mx+1)(2my+1)(2mz+1) window (weights / wsum applied as a convolution);
 * grad += beta * (u - m) / (m + epps), or beta * (u - m) with no_norm.
 * Types 4-6 (the same three means, mirrored twice as far, taken at every
 * voxel's neighbours too): grad += beta * sum_d w_d g(u, M(x + d)) over the
 * window's offsets d (raw weights, x fastest) with g = log(max(u / M,
 * 1e-6)) (4), (u' - M) / u' - ((u' - M) / (sqrt(2) u'))^2 (5), 1 - M / u'
 * (6), u' = max(u, 1e-6); no_norm and epps do not apply.  Types 4-6 need
 * 2 mx <= nx (likewise y, z) and take an (nx+2mx)(ny+2my)(nz+2mz)-float
 * scratch image with cudaMallocAsync on `stream`.
 */
int omb_wmean_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx, int32_t my,
                       int32_t mz, const float *weights, float wsum, int32_t mean_type, float epps, float beta,
                       int32_t no_norm, void *stream);

/*
 * Median root prior gradient (priors.h:4-25, medianFilter3D auxKernels.cl:
 * 981-1027): grad += beta * (u - med) / (med + epps) (no_norm: beta *
 * (u - med)), med the median of the (2mx+1)(2my+1)(2mz+1) neighbourhood of u
 * mirrored at its faces (functions.hpp:216-260).  Windows up to 125 voxels.
 */
int omb_mrp_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx, int32_t my,
                     int32_t mz, float epps, float beta, int32_t no_norm, void *stream);

/*
 * The neighbourhood of the L-filter and FMH priors is the reference's offsets
 * grid (computeOffsets.m): columns over -m..m on every axis, m = Ndx, x
 * fastest; 3 axes when Ndx = Ndy = Ndz (mx = my = mz here), 2 when Ndx = Ndy =
 * 1 and Ndz = 0.  Other windows return OMB_ERR_UNSUPPORTED (the reference's
 * grid does not follow them).  The image is mirrored at its faces
 * (functions.hpp:216-260).
 *
 * L-filter prior gradient (L_filter, priors.h:84-97): s = sum over ranks r of
 * a_l[r] times the window value of rank r (ascending); grad += beta * (u - s)
 * / (s + epps) (no_norm: beta * (u - s)).  a_l (device) has one weight per
 * window value; windows up to 125 values (m <= 2).
 */
int omb_lfilter_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx, int32_t my,
                         int32_t mz, const float *a_l, float epps, float beta, int32_t no_norm, void *stream);

/*
 * FMH prior gradient (FMH, priors.h:54-82): the weighted means along 13 lines
 * through the voxel (4 when nz = 1 or mz = 0; line ii = the grid columns
 * m ii + e (c / m - ii), e = 0..2m, c the centre column) with the column ii
 * of fmh_weights (device, (2m + 1) x lines, column-major), and the voxel's
 * value; med = their median (the mean of the middle two of 14);
 * grad += beta * (u - med) / (med + epps) (no_norm: beta * (u - med)).
 * m <= 8.
 */
int omb_fmh_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, int32_t mx, int32_t my,
                     int32_t mz, const float *fmh_weights, float epps, float beta, int32_t no_norm, void *stream);

/*
 * Anisotropic-diffusion prior gradient (priors.h:226-237): grad += beta *
 * (u - AD(u)) / (AD(u) + epps) (no_norm: beta * (u - AD(u))), AD = `niter`
 * steps of 2-D diffusion of every slice (edges replicated) with time step dt
 * and conductance k: flux 1 exponential exp(-g^2 / k^2), 2 quadratic
 * 1 / (1 + g^2 / k^2); diffusion 1 gradient (Perona-Malik), 2 modified
 * curvature.  The reference calls ArrayFire's anisotropicDiffusion here; this
 * restates the published schemes (ArrayFire's own code is not part of the
 * reference).  Allocates two scratch images stream-ordered.
 */
int omb_ad_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float dt, float k,
                    int32_t niter, int32_t flux, int32_t diffusion, float epps, float beta, int32_t no_norm,
                    void *stream);

/*
 * Non-local regulariser gradient (the NLM kernel, auxKernels.cl:297-620, the
 * image read clamped to its edges as the reference's texture sampler reads
 * it): grad += beta * g(u), g of `type` as omb_recon_params.nlm_type lists,
 * over search[3] (Ndx, Ndy, Ndz) offsets with (2 patch + 1)^3 patches
 * weighted by `gaussian` (device, x fastest) and w = exp(-distance / h);
 * `ref` (device, or NULL) supplies the patches instead of u.  ggmrf_pqc
 * (host, 3 values) only for type 6.  adaptive != 0 (options.NLAdaptive):
 * w = exp(-distance / (distance / patch_voxels * h + adaptive_s)).
 */
int omb_nlm_gradient(const float *u, const float *ref, float *grad, int32_t nx, int32_t ny, int32_t nz,
                     const int32_t *search, const int32_t *patch, const float *gaussian, float h, float epps,
                     float beta, int32_t type, float gamma, const float *ggmrf_pqc, int32_t adaptive,
                     float adaptive_s, void *stream);

/*
 * One relaxed OSEM (ROSEM) sub-iteration (subiterStep.h:137-145,
 * algorithms.h:102-106): the OSEM ratio y / (fp + epps [+ randoms]), its
 * backprojection rhs, then image + lambda * image / sens * (rhs - sens).
 */
int omb_rosem_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const float *sens,
                     float lambda, float *work_meas, float *work_img, void *stream);

/*
 * One RAMLA / BSREM sub-iteration (subiterStep.h:130-135, 232-236;
 * algorithms.h:54-64 on the GPU path): rhs = the backprojection of
 * y / (fp + epps [+ randoms]) - 1 (NaN / Inf -> epps), then
 * image + lambda * rhs * image, clamped to >= epps when `positivity` is set
 * (PoissonUpdate, auxKernels.cl:1997-2026).  No sensitivity image.
 */
int omb_ramla_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, float lambda,
                     int32_t positivity, float *work_meas, float *work_img, void *stream);

/*
 * One PKMA sub-iteration (subiterStep.h:281-295, algorithms.h:151-212
 * without automatic relaxation; image preconditioner as omb_precond_image
 * lists, precond_d its D or NULL with precond 0): rhs = the backprojection
 * of 1 - y / (fp + epps [+ randoms]) (NaN / Inf -> epps) plus du (device,
 * the prior gradient with its weight; NULL: none); x_a = x - lambda * rhs,
 * max(epps, x_a) when `positivity`; image = (1 - alpha) image + alpha x_a.
 */
int omb_pkma_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, float lambda, float alpha,
                    const float *du, int32_t positivity, const float *precond_d, int32_t precond, float *work_meas,
                    float *work_img, void *stream);

/*
 * One MRAMLA / MBSREM sub-iteration (subiterStep.h:123-128, 237-241,
 * algorithms.h:31-52 without preconditioner): rhs = the backprojection of
 * y / (fp + epps [+ randoms]) - 1 plus du (NULL: none, MRAMLA); image +
 * lambda * rhs, max(epps, .) when `positivity`, values >= upper set to
 * upper - epps.  Randoms, when set, must be positive: the reference treats
 * zero-randoms bins with a separate bound (epsilon_mramla) not built here.
 */
int omb_mbsrem_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, float lambda,
                      float upper, const float *du, int32_t positivity, const float *precond_d, int32_t precond,
                      float *work_meas, float *work_img, void *stream);

/*
 * The image preconditioners of PKMA / MRAMLA / MBSREM (applyImagePreconditioning,
 * functions.hpp:2057-2106; the sub-iteration entries take `precond` 0 none,
 * 1 rhs / D (options.precondTypeImage[0]), 2 rhs * x / D ([1]; MBSREM folds x
 * >= U / 2 to U - x)) and their D (device, one image): the subsets' summed
 * A^T 1 divided by the subset count, zeros set to 1 (reconstructionAF.h:
 * 779-816).  work_img: one image of scratch.  PET sinogram data.
 */
int omb_precond_image(omb_handle *h, float *d, float *work_img, void *stream);

/*
 * The MAP step of BSREM and ROSEM-MAP after each iteration (algorithms.h:
 * 130-135): image -= lambda * image * du, then image = max(image, epps);
 * du (device, n voxels) is the prior gradient with its weight.
 */
int omb_map_step(float *image, const float *du, int64_t n, float lambda, float epps, void *stream);

/*
 * PSF blur (Convolution3D_f, auxKernels.cl:192-245): out = window applied at
 * every voxel of `in` (device), the window (device, (2gx+1)(2gy+1)(2gz+1)
 * weights, x fastest; proj.py PSFKernel gives the Gaussian one) read with the
 * image mirrored at its faces, edge voxel repeated.  The reference blurs
 * before the forward projection and after the backprojection.  Not in place.
 */
int omb_psf_convolve(const float *in, float *out, int32_t nx, int32_t ny, int32_t nz, const float *window,
                     int32_t gx, int32_t gy, int32_t gz, void *stream);

/*
 * Relative difference prior gradient (RDPKernel, auxKernels.cl:664-872,
 * 6-neighbour form; neighbours outside the image read 0 as with the CUDA
 * border addressing): grad += beta * dRDP(u)/du with parameters gamma, epps.
 */
int omb_rdp_gradient(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float gamma, float epps,
                     float beta, void *stream);

/*
 * The same with the edge rule chosen: edge 0 reads neighbours outside the
 * image as 0 (omb_rdp_gradient; the reference's buffer path and its
 * util/priors.py RDP), 1 clamps them to the edge voxel (the reference's
 * built-in reconstruction with options.useImages, its default: the prior
 * reads the image through a clamp-to-edge texture, ProjectorClass.h:
 * 6574-6576, samplerRDP auxKernels.cl:653).
 */
int omb_rdp_gradient_ex(const float *u, float *grad, int32_t nx, int32_t ny, int32_t nz, float gamma, float epps,
                        float beta, int32_t edge, void *stream);

/*
 * PET corrections of the projector type-1 forward and backward projections
 * (the reference's NORM, SCATTER, ATNM and ATN kernel options,
 * projectorType123.cl:373-376, 975-987; CPU projector
 * projector_functions.h:1754-1832).  meas_weights: one multiplicative factor
 * per measurement of all subsets in subset order (normalisation x
 * multiplicative scatter x LOR attenuation factors, premultiplied), shared by
 * a measurement's TOF bins; atten_image: attenuation coefficients (1/mm), one
 * per voxel, whose line integral along each ray gives the factor
 * exp(-sum mu x length).  Each ray's factor multiplies its normalisation
 * (1/L x global_factor), so it scales forward projections, backprojections
 * and sensitivity images alike.  Either pointer may be NULL (that correction
 * off); host or device memory, copied into the handle.  Other projector types
 * return OMB_ERR_UNSUPPORTED while corrections are set.
 */
int omb_set_corrections(omb_handle *h, const float *meas_weights, int64_t n_weights, const float *atten_image,
                        int64_t n_atten, void *stream);

/*
 * Randoms (or additive scatter) estimate of the OSEM sub-iterations
 * (omb_osem_subset, omb_osem_subset_frames): the ratio becomes
 * y / (A x + epps + r) (computeForwardProject.h:46-71), r shared by a
 * measurement's TOF bins and by the frames of a batch.  One value per
 * measurement of all subsets in subset order; host or device memory, copied;
 * NULL turns it off.
 */
int omb_set_randoms(omb_handle *h, const float *randoms, int64_t n, void *stream);

/*
 * Device error word of the kernels' bounded waits (TMA and tensor-core
 * pipelines): 0 when no wait ran out since the last call, 1 when one did (the
 * results of that launch are invalid); reading it resets it.  < 0 if the
 * word could not be read.  Synchronises the device.
 */
int omb_take_device_error(void);
int omb_set_tuning(omb_handle *h, const omb_tuning *in);

/*
 * Times each candidate launch shape of the handle's forward and backward
 * projectors over all subsets -- n_frames images at once (type 1 without
 * TOF; otherwise one) with `repeats` timed calls after one warm-up call --
 * and keeps the fastest in the handle (also written to *out unless NULL).
 * Allocates and frees its own scratch buffers on `stream` (about
 * n_frames * (2 images + 1 measurement vector)) and synchronises it; do not
 * call it while `stream` is being captured into a CUDA graph.
 */
int omb_autotune(omb_handle *h, int32_t n_frames, int32_t repeats, omb_tuning *out, void *stream);

/*
 * One PDHG iteration with a TV-gradient term over all projections (one
 * subset), on the device, no host synchronisation:
 *   p      = (p + sigma * (A x - y)) / (1 + sigma)
 *   rhs    = A^T p + beta * gradTV(x)       (smoothed TV, edge-clamped neighbours)
 *   u_new  = max(epps, u - tau * rhs)       (max only when positivity != 0)
 *   x_next = u_new + theta * (u_new - u);   u = u_new
 * x_next must differ from x (the caller swaps them).  work_meas holds
 * omb_measurement_count(h, -1) floats, work_img Nx*Ny*Nz.
 * Restates computeForwardProject.h:227-316 (dual), priors.h:404-409 with
 * TVKernel auxKernels.cl:1733-1990 (TV gradient), algorithms.h:329-420 with
 * PDHGUpdate auxKernels.cl:2034-2062 (primal).
 */
int omb_pdhg_iteration(omb_handle *h, float *x, float *x_next, float *u, float *p, const float *y, float tau,
                       float sigma, float theta, float beta, float tv_smooth, int32_t positivity, float *work_meas,
                       float *work_img, void *stream);

/*
 * The two non-projector steps of omb_pdhg_iteration, for callers that run
 * the projections themselves (omb_forward / omb_backward):
 *   omb_pdhg_dual:   p = (p + sigma * (fp - y)) / (1 + sigma) over n entries
 *                    (computeForwardProject.h:227-316, one subset, no TOF);
 *   omb_pdhg_primal: u_new = max(epps, u - tau * (rhs + beta * gradTV(x))),
 *                    x_next = u_new + theta * (u_new - u), u = u_new, with
 *                    rhs = A^T p (PDHGUpdate auxKernels.cl:2034-2062).
 * omb_forward -> omb_pdhg_dual -> omb_backward -> omb_pdhg_primal is exactly
 * omb_pdhg_iteration.
 */
int omb_pdhg_dual(float *p, const float *fp, const float *y, int64_t n, float sigma, void *stream);
int omb_pdhg_primal(omb_handle *h, const float *x, const float *rhs, float *u, float *x_next, float tau, float theta,
                    float beta, float tv_smooth, int32_t positivity, void *stream);

/*
 * Largest eigenvalue L of A^T A by n_iter power iterations starting from x
 * (unit norm; overwritten with the last iterate).  The PDHG primal step is
 * tau = 1/L with sigma = 1 (functions.hpp:2417-2540, 2886-2905).  `work`
 * holds omb_power_workspace_bytes() bytes.  Synchronises `stream`.
 */
int omb_power_method(omb_handle *h, int32_t n_iter, float *x, float *work_meas, float *work_img, void *work,
                     double *out_host, void *stream);
size_t omb_power_workspace_bytes(void);

/*
 * Poisson log-likelihood sum_i [ y_i * log(fp_i + epps) - (fp_i + epps) ],
 * accumulated in FP64 on the device, written to *out_host.  Synchronises
 * `stream`.  `work` is caller scratch of at least omb_reduce_workspace_bytes(n)
 * bytes.  The reference computes no likelihood; this is the measurement the
 * OSEM comparisons use.
 */
int omb_loglik(const float *y, const float *fp, int64_t n, float epps, double *out_host,
               void *work, void *stream);
size_t omb_reduce_workspace_bytes(int64_t n);

/*
 * Largest image (voxels) omb_backward_fixed64_noalloc accepts.  Its int64
 * scratch is a fixed array of 2 * OMB_NOALLOC_MAX_VOXELS * 8 bytes (16 MiB)
 * in device memory of every GPU that loads this library, held until exit.
 */
#define OMB_NOALLOC_MAX_VOXELS (1u << 20)

/*
 * Int64 fixed-point backprojection (projector type 1) that allocates nothing,
 * for callers that cannot call cudaMalloc -- their device memory belongs to
 * another allocator (a framework's caching pool, or a pipeline that fixes its
 * memory budget at start-up).  No counterpart in the reference: it is the
 * allocation-free form of omb_backward(..., OMB_BP_FIXED64, ...) and gives
 * the same result.
 * No handle: `desc` is the same descriptor as for omb_create, except that
 * the per-ray geometry is already on the device: desc->xy, desc->z and
 * desc->tof_centers are DEVICE pointers, while desc->n_meas stays a HOST
 * array (it is read on the host to size the launch).  y, image and sens (may
 * be NULL) are device buffers; image and sens are overwritten.  Images above OMB_NOALLOC_MAX_VOXELS voxels are
 * rejected with OMB_ERR_UNSUPPORTED.
 * The scratch array is shared by all calls and keeps the last call's
 * contents (each call clears what it uses); calls that overlap on the GPU
 * (different streams or threads on one device) race on it.  The first call
 * on each device looks up the array's device address (cudaGetSymbolAddress)
 * and caches it; make that first call before any stream capture.  The
 * cached address belongs to the device's primary context: calls after
 * cudaDeviceReset on that device are not supported.
 */
int omb_backward_fixed64_noalloc(const omb_geometry_desc *desc, int32_t subset, const float *y, float *image,
                                 float *sens, void *stream);

/*
 * Batches of independent CT reconstructions -- e.g. 2-D fan-beam slices of
 * different image sizes and view counts -- projected by ONE persistent
 * launch per direction instead of one launch per item.  Every item is a CT
 * geometry with projector type 1 and no TOF; all of its projections are
 * projected (subset order).  Images of all items are concatenated in one
 * float buffer (item i starts at omb_batch_image_offset(b, i)), measurements
 * likewise (omb_batch_measurement_offset); offset n is the total.  The
 * reference launches one kernel per reconstruction object (projfunctions.py:
 * 86, 735); this has no counterpart there.
 */
typedef struct omb_batch omb_batch;
int omb_batch_create(const omb_geometry_desc *descs, int32_t n, omb_batch **out);
int omb_batch_destroy(omb_batch *b);
int64_t omb_batch_image_offset(const omb_batch *b, int32_t item);
int64_t omb_batch_measurement_offset(const omb_batch *b, int32_t item);
/* y = A images for every item (y overwritten). */
int omb_batch_forward(omb_batch *b, const float *images, float *y, void *stream);
/* images = A^T y for every item (images overwritten). */
int omb_batch_backward(omb_batch *b, const float *y, float *images, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* OMEGA_B200_H */
