// Internal launchers shared between the kernel files and the C-ABI layer.
#pragma once

#include "common.cuh"

namespace omb {

int siddon_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, const Tuning &tn,
                   cudaStream_t st);
int siddon_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, float *sens,
                    const Tuning &tn, cudaStream_t st);
int siddon_backward_fixed(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y,
                          unsigned long long *acc, unsigned long long *acc_sens, cudaStream_t st);
int siddon_count(const Grid &g, const RaySet &rs, const Tof &tof, unsigned long long *total, cudaStream_t st);
int fixed_to_float(const unsigned long long *acc, float *out, int64_t n, cudaStream_t st);

// Subset count and image grid of a handle (the handle layout is private to api.cu).
int handle_subsets(const omb_handle *h);
Grid handle_grid(const omb_handle *h);
float handle_epps(const omb_handle *h);
// du = beta * clamp(du, -delta, delta)
int scale_clamp(float *du, int64_t n, float beta, float delta, cudaStream_t st);
// x = x / (sens + du) * rhs
int osl_update(float *img, const float *sens, const float *du, const float *rhs, int64_t n, cudaStream_t st);

// Relaxation of one sub-iteration: lam[*iter] from a device schedule (the
// built-in loop, so a captured iteration replays with the next value), else
// the host value v.
struct Relax {
    const float *lam = nullptr;
    const int *iter = nullptr;
    float v = 1.f;
};
// PKMA momentum of one sub-iteration: alpha[*iter * n_subsets + subset] from
// a device schedule, else the host value v.
struct Momentum {
    const float *alpha = nullptr;
    const int *iter = nullptr;
    int n_subsets = 1;
    int subset = 0;
    float v = 1.f;
};
// fp = sign * (y / ((fp + epps) [+ r]) - shift), NaN / Inf -> epps; r (nullable) per ray, shared by TOF bins
int ratio_shift(const float *y, float *fp, int64_t n, const float *rnd, int64_t n_rays, float epps, float shift,
                float sign, cudaStream_t st);
// ROSEM: x = x + lam * x / sens * (rhs - sens)
int rosem_update(float *img, const float *sens, const float *rhs, int64_t n, Relax lam, cudaStream_t st);
// RAMLA / BSREM: x = x + lam * rhs * x, then max(epps, x) when positivity
int bsrem_update(float *img, const float *rhs, int64_t n, Relax lam, float epps, bool positivity, cudaStream_t st);
// PKMA: g = rhs [+ du]; xa = x - lam * g, max(epps, xa) when positivity; x = (1 - a) x + a xa
int pkma_update(float *img, const float *rhs, const float *du, int64_t n, Relax lam, Momentum a, float epps,
                bool positivity, const float *dd, int mode, cudaStream_t st);
// MRAMLA / MBSREM: x = x + lam * (rhs [+ du]), max(epps, x) when positivity, x >= U -> U - epps
int mbsrem_update(float *img, const float *rhs, const float *du, int64_t n, Relax lam, float epps, float upper,
                  bool positivity, const float *dd, int mode, cudaStream_t st);
// PKMA / MBSREM image preconditioning: D = sum / S with zeros -> 1; acc += v
int precond_finish(float *dd, int64_t n, int subsets, cudaStream_t st);
int add_into(float *acc, const float *v, int64_t n, cudaStream_t st);
// A^T 1 of one subset without the epps floor of omb_sensitivity
int sensitivity_raw(omb_handle *h, int32_t subset, float *sens, cudaStream_t st);
// MAP step: x = x - lam * x * du, then max(epps, x)
int map_step(float *img, const float *du, int64_t n, Relax lam, float epps, cudaStream_t st);
// ++*iter on the stream
int relax_advance(int *iter, cudaStream_t st);
// The relaxed sub-iterations of a handle.
enum RelaxedKind { kRosem = 0, kRamla = 1, kPkma = 2, kMbsrem = 3 };
// The other image preconditioners of PKMA / MRAMLA / MBSREM (elementwise.cu): the gradient times the type-4
// image gradF (from sub-iteration grad_init on), the type-3 value alpha[k], the types 0 / 1 / 2 factor
// (mode 1: 1 / D, 2: xp / D, 3: max(xp, max(1e-5, ref)) / D) and the type-6 image dP; k = *it * n_sub + sub,
// xp the image (folded to U - x where x >= U / 2 when fold).
struct PrecondExt {
    int mode = 0;
    const float *dd = nullptr, *ref = nullptr;
    const float *gradF = nullptr;
    int grad_init = 0, grad_last = 0, deriv_type = 0;
    float grad_v1 = 0.5f, grad_v2 = 2.5f;
    const float *alpha = nullptr;
    const float *dP = nullptr;
    const int *it = nullptr;
    int n_sub = 1, sub = 0;
    int fold = 0;
    float upper = 10000.f;
    // type 5: the image filter's taps (or NULL), length, filtering sub-iterations and scratch image
    const float *filt_h = nullptr;
    int filt_nf = 0, filt_K = 0;
    float *filt_tmp = nullptr;
};
struct RelaxedArgs {
    int kind = kRosem;
    const float *sens = nullptr;   // ROSEM
    const float *du = nullptr;     // PKMA / MBSREM: prior gradient (weight included) added to the gradient, or NULL
    Relax lam;
    Momentum alpha;                // PKMA
    float upper = 10000.f;         // MRAMLA / MBSREM: U
    bool positivity = true;
    const float *precond_d = nullptr;  // PKMA / MBSREM: D of the image preconditioner
    int precond = 0;               // 0 none, 1 g / D (type 0), 2 g * x / D (type 1)
    // the other preconditioners (when ext_on): applied by precond_apply before the update, which then
    // takes the gradient as it is
    bool ext_on = false;
    PrecondExt ext;
    float *gradF = nullptr;        // type-4 image, recomputed in its window
    double *work = nullptr;        // precond_workspace_bytes() + 2 dot2 workspaces (type 4, relaxation)
    const float *meas_m = nullptr; // measurement preconditioner type 0: the subset's A 1 (zeros -> 1), or NULL
    bool auto_relax = false, relax_scaling = false;  // PKMA: lam from the norms (needs lam.lam)
};
int relaxed_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const RelaxedArgs &a,
                   float *work_meas, float *work_img, cudaStream_t st);

int precond_apply(float *g, const float *du, const float *img, int64_t n, const PrecondExt &p, cudaStream_t st);
// Type 4: recomputes gradF from img when the sub-iteration lies in [grad_init, grad_last] (device-side check).
size_t precond_workspace_bytes();
int precond_gradient(const float *img, float *gradF, const Grid &g, const PrecondExt &p, double *work,
                     cudaStream_t st);
// PKMA's automatic relaxation / relaxation scaling of lam[*it] from dot2 results (x.g, g.g) and (g.x, x.x).
int pkma_relax(float *lam, const int *it, int sub, const double *xg_gg, const double *gx_xx, bool compute,
               bool scaling, cudaStream_t st);
int div_inplace(float *a, const float *b, int64_t n, cudaStream_t st);
int curv_meas(float *e, const float *y, int64_t n, cudaStream_t st);
int curv_acc(float *dp, const float *rhs, int64_t n, int subsets, bool first, cudaStream_t st);
int curv_finish(float *dp, int64_t n, cudaStream_t st);
int zero_to_one(float *a, int64_t n, cudaStream_t st);

// Projector types 2 / 3 (PET), one frame.
int orth_forward(const Grid &g, const RaySet &rs, const Orth &o, const Tof &tof, float gf, const float *img, float *y,
                 cudaStream_t st);
int orth_backward(const Grid &g, const RaySet &rs, const Orth &o, const Tof &tof, float gf, const float *y, float *img,
                  float *sens, cudaStream_t st);
// The tube tracer's count and fill passes of the transposed system matrix (non-TOF; sysmat_build).
// rcnt: each ray's entry count; rsoff / rsent (or NULL): the ray-major copy in slices of 32 rays.
int orth_sm_count(const Grid &g, const RaySet &rs, const Orth &o, float gf, unsigned *cnt, unsigned *rcnt,
                  cudaStream_t st);
int orth_sm_fill(const Grid &g, const RaySet &rs, const Orth &o, float gf, unsigned long long *cursor, uint2 *ent,
                 const int64_t *rsoff, uint2 *rsent, cudaStream_t st);

// Multi-ray PET projections (rs.nr_xy x rs.nr_z rays per LOR), one frame.
int multiray_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *img, float *y,
                     int per_sm, cudaStream_t st);
int multiray_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y, float *img,
                      float *sens, int per_sm, cudaStream_t st);

// Projector type 5 (branchless distance-driven), CT.
int bdd_forward(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                int64_t nproj, const float *img, float *imgT, float *y, const Tuning &tn, cudaStream_t st);
// The same projection with per-slice image boxes staged by TMA (cols = 8 or 16 columns per thread; the same
// numbers as bdd_forward with bdd_fp_cols = cols).
bool bdd_fp_tma_supported(const Grid &g, const float *img, const float *imgT);
int bdd_forward_tma(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                    int64_t nproj, const float *img, const float *imgT, float *y, int cols, cudaStream_t st);
// Device error word of the bounded waits (1 after a wait ran out; reset when read), < 0 on failure.
int take_device_error();
int bdd_backward(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj, const float *y,
                 float *img, float *sens, const Tuning &tn, cudaStream_t st);
// Ray-driven (scatter) type-5 backprojection, the exact adjoint of the forward
// projection: float atomics into img / sens (zeroed by the caller), or int64
// fixed-point atomics into acc / acc_s (when acc is not NULL).
int bdd_backward_ray(const Grid &g, const float *xy, const float *uv, int nr, int nc, float pitch_y, int64_t proj0,
                     int64_t nproj, const float *y, float *img, float *sens, unsigned long long *acc,
                     unsigned long long *acc_s, cudaStream_t st);
// The same backprojection with per-projection detector boxes staged by TMA (kz = 8 or 16 voxels along z per
// thread; the same numbers as bdd_backward with bdd_bp_z = kz).
bool bdd_bp_tma_supported(int nr, const float *y);
int bdd_backward_tma(const Grid &g, const BddProj *pj, const BddMap64 *pm, int nr, int nc, int64_t nproj,
                     const float *y, float *img, float *sens, int kz, cudaStream_t st);

// Resident transposed system matrix of the type-1 non-TOF projector for one subset (sysmat.cu): for each
// voxel the (ray, weight) pairs of the rays crossing it, in ray order; off[v] .. off[v + 1] index ent.
struct SysMat {
    int64_t proj0 = 0, m_size = 0;
    int cur_subset = 0;
    int64_t *off = nullptr;
    uint2 *ent = nullptr;  // (launch-local ray index, weight bits), voxel-major lists
    int64_t nnz = 0;
    // sliced copy (when it fits): slices of 32 consecutive voxels, entry k of the slice's voxel l at
    // soff[slice] + 32 k + l; the voxel-major lists are released once it is built
    int64_t *soff = nullptr;
    uint2 *sent = nullptr;
    // tube weights only: the ray-major copy for the forward projection (slices of 32 rays, entry k of ray l
    // at rsoff[slice] + 32 k + l, (voxel, weight bits)) and each ray's entry count; NULL when it did not fit
    int64_t *rsoff = nullptr;
    uint2 *rsent = nullptr;
    unsigned *rcnt = nullptr;
};
// Builds sm for the rays of rs (the walk and weights of the ray-driven backprojection: the Siddon tracer, or
// with `orth` the non-TOF tube tracer of projector types 2 / 3); synchronises `st` and refuses to run while
// `st` is captured into a CUDA graph.
int sysmat_build(const Grid &g, const RaySet &rs, float gf, SysMat &sm, cudaStream_t st, const Orth *orth = nullptr);
void sysmat_free(SysMat &sm);
// Backprojection of fr.n frames through sm (images overwritten); ym: ray-major scratch of at least
// 8 * m floats (4 * m for 4..7 frames; unused for fewer).
int sysmat_backward(const Grid &g, const SysMat &sm, const Frames &fr, int64_t m, float *ym, int64_t ym_floats,
                    cudaStream_t st);
// Forward projection of fr.n frames through sm's ray-major copy (types 2 / 3; sm.rsent != NULL).
int sysmat_forward(const Grid &g, const SysMat &sm, const Frames &fr, int64_t m, cudaStream_t st);

// Detector-row filtering (filter.cu): out = the circular convolution (length nf) of each column of nr rows with
// h; the measurement residual fp -= y; the dual step out = (p + sigma r) / denom (denom 1: no division).
int circ_filter(const float *in, float *out, int nr, int64_t ncols, const float *h, int nf, cudaStream_t st);
// The filtering-based image preconditioner: g (nx x ny x nz) filtered slice by slice with the separable
// circular filter h (x lines into tmp, then y lines back into g); with a gate counter, only in the
// sub-iterations kk = *it * n_sub + sub < K (K > 0) or kk == 0 (K == 0), g untouched otherwise.
struct FilterGate {
    const int *it = nullptr;
    int n_sub = 1, sub = 0, K = 0;
};
int image_filter(float *g, float *tmp, int nx, int ny, int nz, const float *h, int nf, const FilterGate &gate,
                 cudaStream_t st);
int meas_residual(float *fp, const float *y, int64_t n, cudaStream_t st);
int dual_step(const float *p, const float *r, float *out, int64_t n, float sigma, float denom, cudaStream_t st);

// Projector type 4 (interpolation), PET and CT.
int interp_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, float dL, const float *img,
                   const __nv_bfloat16 *img16, float *y, const Tuning &tn, cudaStream_t st);
// BF16 copy of n floats (also the network's weight conversion).
int unet_to_bf16(const float *a, void *b, int64_t n, cudaStream_t st);
int interp_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, float dL, const float *y, float *img,
                    float *sens, unsigned long long *acc, unsigned long long *acc_s, const Tuning &tn,
                    cudaStream_t st);
int interp_ct_backward(const Grid &g, const BddProj *pj, int nr, int nc, int64_t nproj, float kerroin,
                       const float *y, float *img, float *sens, cudaStream_t st);

// Batches of independent CT geometries in one persistent launch (batch.cu).
int batch_project(const BatchItem *items, const int2 *work, int n_work, int *counter, const float *in, float *out,
                  bool backward, cudaStream_t st);

// PDHG + TV and the power method.
int pdhg_dual(float *p, const float *fp, const float *y, int64_t n, float sigma, cudaStream_t st);
int pdhg_primal_tv(const Grid &g, const float *x, const float *rhs, float *u, float *x_out, float beta, float smooth,
                   float tau, float theta, float epps, int positivity, cudaStream_t st);
size_t dot_workspace_bytes();
int dot2(const float *a, const float *b, int64_t n, double *work, cudaStream_t st);
int normalize_into(float *x, const float *b, int64_t n, const double *dots, cudaStream_t st);

// Elementwise steps of the subset updates.
int osem_ratio(const float *y, float *fp, int64_t n, float epps, cudaStream_t st);
// y / (fp + epps + randoms[i % n_rays]) for `frames` frames sharing the randoms
int osem_ratio_randoms(const float *y, int64_t y_stride, float *fp, int64_t fp_stride, int64_t n, int frames,
                       const float *rnd, int64_t n_rays, float epps, cudaStream_t st);
int em_update(float *img, const float *sens, const float *rhs, int64_t n, float epps, cudaStream_t st);
int clamp_min(float *x, int64_t n, float lo, cudaStream_t st);
int osem_ratio_frames(const float *y, int64_t y_stride, float *fp, int64_t fp_stride, int64_t n, int frames,
                      float epps, cudaStream_t st);
int em_update_frames(float *img, int64_t img_stride, const float *sens, const float *rhs, int64_t rhs_stride,
                     int64_t n, int frames, float epps, cudaStream_t st);
size_t reduce_workspace_bytes(int64_t n);
int loglik(const float *y, const float *fp, int64_t n, float epps, double *out_host, void *work,
           cudaStream_t st);

}  // namespace omb
