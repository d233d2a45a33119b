// C-ABI entry points (include/omega_b200.h): handle life cycle, argument
// validation and dispatch to the projector kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"

namespace omb {

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return set_error(OMB_ERR_CUDA, m);
}

}  // namespace omb

using namespace omb;

struct omb_handle {
    int device = 0;
    omb_geometry_desc desc{};
    std::vector<int64_t> n_meas;  // cumulative sinograms/projections per subset
    Grid grid{};
    Tof tof{};
    float *d_xy = nullptr;
    uint16_t *d_tr = nullptr;             // index-based events: transaxial / axial index pairs
    uint16_t *d_ax = nullptr;
    float *d_z = nullptr;
    float *d_tofc = nullptr;
    unsigned long long *d_acc = nullptr;  // 2 * N int64 accumulators (fixed-point BP)
    float *d_imgT = nullptr;              // y-fastest image copy (type-5 forward projection)
    BddProj *d_bddp = nullptr;            // per-projection maps (type-5 backprojection)
    BddMap64 *d_bddm64 = nullptr;         // the same maps in FP64 (re-based per block by the type-5 backprojection)
    int64_t n_img = 0;
    Tuning tune{};
    int read_mode = OMB_READ_FP32;        // image precision of the type-1/4 forward projections
    __nv_bfloat16 *d_img16 = nullptr;     // BF16 image copies (read_mode == OMB_READ_BF16)
    int img16_frames = 0;                 // frames d_img16 holds
    std::vector<SysMat> sysmats;          // type-1 transposed system matrices, one per subset used
    float *d_ym = nullptr;                // ray-major measurement scratch of the system-matrix backprojection
    int64_t ym_floats = 0;
    float *d_ilv = nullptr;               // voxel-interleaved frame scratch (type-1 frame batches)
    int64_t ilv_floats = 0;               // its capacity
    float *d_w = nullptr;                 // PET: multiplicative weight per measurement (all subsets), or NULL
    float *d_mu = nullptr;                // PET: attenuation image, or NULL
    float *d_rand = nullptr;              // PET: randoms per measurement (all subsets) for the OSEM ratio, or NULL
    float *d_vol = nullptr;               // type 3: the intersection-volume table
    Orth orth_fp{}, orth_bp{};            // types 2 / 3: the tube of the forward / backward projector
    // Buffers replaced by larger ones.  They are freed only with the handle:
    // a CUDA graph captured earlier may still address them.
    std::vector<void *> retired;
};

// Attaches the voxel-interleaved scratch to a type-1 frame batch, growing it
// to ceil(n / 8) * 8 images when needed.  Growing allocates, so it is skipped
// while the stream is being captured into a CUDA graph: the batch then takes
// the frame-major kernels (the capture's warm-up call normally grew it).
static void attach_interleave(omb_handle *h, Frames &f, cudaStream_t s) {
    f.ilv = nullptr;
    f.ilv_floats = 0;
    if (h->tune.siddon_layout != 1 || h->desc.tof_bins != 1 || f.n < 4) return;
    const int64_t need = (int64_t)((f.n + 7) / 8) * 8 * h->n_img;
    if (need > h->ilv_floats) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
        float *p = nullptr;
        if (cudaMalloc(&p, (size_t)need * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();  // out of memory: keep the frame-major kernels
            return;
        }
        if (h->d_ilv) h->retired.push_back(h->d_ilv);
        h->d_ilv = p;
        h->ilv_floats = need;
    }
    f.ilv = h->d_ilv;
    f.ilv_floats = h->ilv_floats;
}

// Type-5 backprojection maps of every projection, FP64 on the host from the
// same vectors the reference's computeGeom5 uses (omegatomo/projector/
// init.py:6-37): panel corner d3 = d - apuX - apuY, unit axes along apuX and
// apuY, plane normal cross(apuX - apuY, -apuX - apuY).
static std::vector<BddProj> bdd_maps(const omb_geometry_desc &d, std::vector<BddMap64> *maps64 = nullptr) {
    std::vector<BddProj> out((size_t)d.n_proj);
    if (maps64) maps64->assign((size_t)d.n_proj, BddMap64{});
    const double nr2 = (double)d.n_rows_d / 2.0, nc2 = (double)d.n_cols_d / 2.0;
    for (int64_t p = 0; p < d.n_proj; ++p) {
        const float *q = d.xy + p * 6;
        const double s[3] = {q[0], q[1], q[2]}, dd[3] = {q[3], q[4], q[5]};
        const double ax[3] = {d.z[p * 2] * nr2, d.z[p * 2 + 1] * nr2, 0.0};
        const double ay[3] = {0.0, 0.0, nc2 * (double)d.dpitch_y};
        double d3[3], d2[3], e[3];
        for (int k = 0; k < 3; ++k) {
            d3[k] = dd[k] - ax[k] - ay[k];
            d2[k] = ax[k] - ay[k];
            e[k] = -ax[k] - ay[k];
        }
        double n[3] = {d2[1] * e[2] - d2[2] * e[1], d2[2] * e[0] - d2[0] * e[2], d2[0] * e[1] - d2[1] * e[0]};
        const double nl = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double lx = sqrt(ax[0] * ax[0] + ax[1] * ax[1]), ly = fabs(ay[2]);
        const double ex[3] = {ax[0] / lx, ax[1] / lx, 0.0}, ey[3] = {0.0, 0.0, ay[2] / ly};
        for (int k = 0; k < 3; ++k) n[k] /= nl;
        auto dot = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
        const double sd[3] = {s[0] - d3[0], s[1] - d3[1], s[2] - d3[2]};
        const double A = dot(ex, sd), Av = dot(ey, sd), B = -dot(n, sd);
        const double D0 = -dot(n, s);  // n.(q - s) at q = 0
        BddProj P{};
        double cu[3], cv[3];
        for (int k = 0; k < 3; ++k) {
            cu[k] = A * n[k] + B * ex[k];
            cv[k] = Av * n[k] + B * ey[k];
        }
        for (int k = 0; k < 3; ++k) {
            P.au[k] = (float)(cu[k] / ((double)d.dpitch_x * D0));
            P.av[k] = (float)(cv[k] / ((double)d.dpitch_y * D0));
            P.c[k] = (float)(n[k] / D0);
            P.s[k] = (float)s[k];
        }
        P.au0 = (float)(-dot(cu, s) / ((double)d.dpitch_x * D0));
        P.av0 = (float)(-dot(cv, s) / ((double)d.dpitch_y * D0));
        if (maps64) {
            BddMap64 &M = (*maps64)[(size_t)p];
            for (int k = 0; k < 3; ++k) {
                M.au[k] = cu[k] / ((double)d.dpitch_x * D0);
                M.av[k] = cv[k] / ((double)d.dpitch_y * D0);
                M.c[k] = n[k] / D0;
            }
            M.au0 = -dot(cu, s) / ((double)d.dpitch_x * D0);
            M.av0 = -dot(cv, s) / ((double)d.dpitch_y * D0);
        }
        P.ysl = fabs(s[0]) <= fabs(s[1]);
        P.spos = P.ysl ? (s[1] > 0.0) : (s[0] > 0.0);
        const double dms[3] = {dd[0] - s[0], dd[1] - s[1], dd[2] - s[2]};
        P.k = (float)(dot(n, dms) / D0);
        out[(size_t)p] = P;
    }
    return out;
}

// Measurement-level subsets (types 1, 2, 4, 5) of sinogram data; list-mode
// events arrive already in subset order and split into contiguous ranges.
static bool meas_level_subsets(const omb_geometry_desc &d) {
    return d.n_subsets > 1 && d.subset_type < 8 && d.modality == OMB_PET_SINOGRAM;
}

static int validate(const omb_geometry_desc *d) {
    if (!d) return set_error(OMB_ERR_INVALID, "geometry descriptor is NULL");
    if (d->struct_size != sizeof(omb_geometry_desc))
        return set_error(OMB_ERR_INVALID, "omb_geometry_desc.struct_size does not match this library (" +
                                              std::to_string(sizeof(omb_geometry_desc)) + " bytes)");
    if (d->abi_version != OMB_ABI_VERSION) return set_error(OMB_ERR_INVALID, "unsupported abi_version");
    if (d->modality < OMB_PET_SINOGRAM || d->modality > OMB_PET_INDEXED)
        return set_error(OMB_ERR_INVALID, "unknown modality");
    const bool events = d->modality == OMB_PET_LISTMODE || d->modality == OMB_PET_INDEXED;
    if (events) {
        if (d->n_rows_d != 1 || d->n_cols_d != 1)
            return set_error(OMB_ERR_INVALID, "list-mode data: n_rows_d and n_cols_d must be 1");
        if (d->tof_bins > 1) return set_error(OMB_ERR_UNSUPPORTED, "TOF list-mode data is not built");
        if (d->modality == OMB_PET_INDEXED && (!d->tr_index || !d->ax_index))
            return set_error(OMB_ERR_INVALID, "index-based data needs tr_index and ax_index");
    }
    if (d->fp_type < 1 || d->fp_type > 5)
        return set_error(OMB_ERR_UNSUPPORTED, "forward projector type " + std::to_string(d->fp_type) + " is not built");
    if (d->bp_type < 1 || d->bp_type > 5)
        return set_error(OMB_ERR_UNSUPPORTED, "backprojector type " + std::to_string(d->bp_type) + " is not built");
    const bool orth = d->fp_type == 2 || d->fp_type == 3 || d->bp_type == 2 || d->bp_type == 3;
    if (orth) {
        if (d->modality == OMB_CT_PANEL) return set_error(OMB_ERR_UNSUPPORTED, "projector types 2 / 3 are built for PET");
        if ((d->fp_type == 2 || d->fp_type == 3) && (d->bp_type == 2 || d->bp_type == 3) && d->fp_type != d->bp_type)
            return set_error(OMB_ERR_UNSUPPORTED, "projector types 23 / 32 are not built");
        if (d->nx != d->ny || d->dx != d->dy || d->bx != d->by)
            return set_error(OMB_ERR_UNSUPPORTED,
                             "projector types 2 / 3 need a square transaxial grid (nx == ny, dx == dy, bx == by)");
        if ((d->fp_type == 2 || d->bp_type == 2) && !(d->tube_width > 0.f))
            return set_error(OMB_ERR_INVALID, "projector type 2 needs tube_width (options.tube_width_z) > 0");
        if ((d->fp_type == 2 || d->bp_type == 2) && d->tof_bins > 1)
            return set_error(OMB_ERR_INVALID, "TOF is not supported with projector type 2");
        if (d->fp_type == 3 || d->bp_type == 3) {
            if (!(d->tube_radius > 0.f)) return set_error(OMB_ERR_INVALID, "projector type 3 needs tube_radius > 0");
            if (!d->vol_v || d->n_vol_v < 1 || d->n_vol_v > (1 << 24))
                return set_error(OMB_ERR_INVALID, "projector type 3 needs its volume table vol_v");
            if (!(d->vol_bmax > d->vol_bmin)) return set_error(OMB_ERR_INVALID, "projector type 3 needs vol_bmax > vol_bmin");
        }
    }
    if ((d->fp_type == 5 || d->bp_type == 5) && d->modality != OMB_CT_PANEL)
        return set_error(OMB_ERR_INVALID, "Projector type 5 is only supported with CT data!");
    if ((d->fp_type == 5 || d->bp_type == 5) && d->tof_bins > 1)
        return set_error(OMB_ERR_INVALID, "projector type 5 has no TOF");
    if ((d->fp_type == 4 || d->bp_type == 4) && !(d->dL > 0.f))
        return set_error(OMB_ERR_INVALID, "projector type 4 needs a positive sampling length dL");
    if (d->bp_type == 4 && d->modality == OMB_CT_PANEL && !(d->kerroin > 0.f))
        return set_error(OMB_ERR_INVALID, "the type-4 CT backprojection needs its weight kerroin > 0");
    if (d->n_rays_xy < 0 || d->n_rays_z < 0 || d->n_rays_xy > 64 || d->n_rays_z > 64)
        return set_error(OMB_ERR_INVALID, "rays per LOR must be in 0..64");
    if (std::max(d->n_rays_xy, 1) * std::max(d->n_rays_z, 1) > 1) {
        if (d->modality == OMB_CT_PANEL) return set_error(OMB_ERR_UNSUPPORTED, "multi-ray projection is PET-only");
        if (d->fp_type != 1 || d->bp_type != 1)
            return set_error(OMB_ERR_UNSUPPORTED, "multi-ray projection is built for projector type 1");
        if (!(d->dpitch_x > 0.f) || !(d->dpitch_y > 0.f))
            return set_error(OMB_ERR_INVALID, "multi-ray projection needs the crystal pitches dpitch_x, dpitch_y");
    }
    if (d->nx == 0 || d->ny == 0 || d->nz == 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    if (!(d->dx > 0.f) || !(d->dy > 0.f) || !(d->dz > 0.f)) return set_error(OMB_ERR_INVALID, "voxel size must be positive");
    if (d->n_rows_d == 0 || d->n_cols_d == 0) return set_error(OMB_ERR_INVALID, "detector size must be positive");
    if (d->n_proj <= 0) return set_error(OMB_ERR_INVALID, "n_proj must be positive");
    if (d->n_subsets < 1) return set_error(OMB_ERR_INVALID, "n_subsets must be >= 1");
    if (!d->n_meas) return set_error(OMB_ERR_INVALID, "n_meas is NULL");
    if (!d->xy || (!d->z && d->modality != OMB_PET_LISTMODE))
        return set_error(OMB_ERR_INVALID, "xy/z coordinate arrays are NULL");
    // list-mode events come in subset order: contiguous ranges, like whole sinograms
    const bool meas_level = d->n_subsets > 1 && d->subset_type < 8 && !events;
    if (meas_level) {
        if (d->modality != OMB_PET_SINOGRAM)
            return set_error(OMB_ERR_UNSUPPORTED, "measurement-level subset types are PET-only");
        if (d->subset_type != 1 && d->subset_type != 2 && d->subset_type != 4 && d->subset_type != 5)
            return set_error(OMB_ERR_UNSUPPORTED, "subset type " + std::to_string(d->subset_type) + " is not built");
    }
    const int64_t nbin = (int64_t)d->n_rows_d * d->n_cols_d;
    if (d->modality == OMB_PET_SINOGRAM) {
        if (d->n_xy != nbin * 4) return set_error(OMB_ERR_INVALID, "PET xy must hold 4 floats per sinogram bin");
        if (d->n_z != d->n_proj * 2) return set_error(OMB_ERR_INVALID, "PET z must hold 2 floats per sinogram");
    } else if (d->modality == OMB_CT_PANEL) {
        if (d->n_xy != d->n_proj * 6) return set_error(OMB_ERR_INVALID, "CT xy must hold 6 floats per projection");
        if (d->n_z != d->n_proj * 2) return set_error(OMB_ERR_INVALID, "CT z must hold 2 floats per projection");
    } else if (d->modality == OMB_PET_LISTMODE) {
        if (d->n_xy != d->n_proj * 6) return set_error(OMB_ERR_INVALID, "list-mode xy must hold 6 floats per event");
    } else {
        if (d->n_xy < 2 || d->n_xy % 2 || d->n_z < 1)
            return set_error(OMB_ERR_INVALID, "index-based data needs the crystal table (2 floats each) and z");
        // every index must address the tables: checked here once instead of in the kernels
        for (int64_t e = 0; e < 2 * d->n_proj; ++e)
            if ((int64_t)d->tr_index[e] * 2 + 1 >= d->n_xy || (int64_t)d->ax_index[e] >= d->n_z)
                return set_error(OMB_ERR_INVALID, "event " + std::to_string(e / 2) + ": detector index out of range");
    }
    if (d->tof_bins < 1) return set_error(OMB_ERR_INVALID, "tof_bins must be >= 1");
    if (d->tof_bins > kMaxTofBins) return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    if (d->tof_bins > 1) {
        if (!d->tof_centers) return set_error(OMB_ERR_INVALID, "tof_centers is NULL");
        if (!(d->sigma_x > 0.f)) return set_error(OMB_ERR_INVALID, "TOF sigma must be positive");
        if (d->modality == OMB_CT_PANEL) return set_error(OMB_ERR_INVALID, "TOF is PET-only");
    }
    const int64_t *nm = d->n_meas;
    if (nm[0] != 0) return set_error(OMB_ERR_INVALID, "n_meas[0] must be 0");
    for (int s = 0; s < d->n_subsets; ++s)
        if (nm[s + 1] < nm[s]) return set_error(OMB_ERR_INVALID, "n_meas must be non-decreasing");
    if (!meas_level && nm[d->n_subsets] != d->n_proj)
        return set_error(OMB_ERR_INVALID, "n_meas[n_subsets] must equal n_proj");
    return OMB_OK;
}

// Rays of one call: a subset, or every subset when subset == -1.
static int ray_set(const omb_handle *h, int32_t subset, RaySet &rs) {
    const omb_geometry_desc &d = h->desc;
    if (subset < -1 || subset >= d.n_subsets)
        return set_error(OMB_ERR_INVALID, "subset " + std::to_string(subset) + " out of range");
    rs.xy = h->d_xy;
    rs.z = h->d_z;
    rs.tr = h->d_tr;
    rs.ax = h->d_ax;
    rs.modality = d.modality;
    rs.n_rows = (int)d.n_rows_d;
    rs.n_cols = (int)d.n_cols_d;
    rs.pitch_x = d.dpitch_x;
    rs.pitch_y = d.dpitch_y;
    rs.n_subsets = d.n_subsets;
    const int64_t nbin = (int64_t)d.n_rows_d * d.n_cols_d;
    const bool meas_level = meas_level_subsets(d);
    if (meas_level) {
        if (subset < 0) return set_error(OMB_ERR_UNSUPPORTED, "subset -1 needs a whole-sinogram subset type");
        rs.stype = d.subset_type;
        rs.cur_subset = subset;
        rs.proj0 = 0;
        rs.n_proj = d.n_proj;
        rs.m_size = h->n_meas[subset + 1] - h->n_meas[subset];
    } else {
        rs.stype = 0;
        rs.cur_subset = subset < 0 ? 0 : subset;
        rs.proj0 = subset < 0 ? 0 : h->n_meas[subset];
        rs.n_proj = subset < 0 ? d.n_proj : h->n_meas[subset + 1] - h->n_meas[subset];
        rs.m_size = rs.n_proj * nbin;
    }
    rs.nr_xy = std::max(d.n_rays_xy, 1);
    rs.nr_z = std::max(d.n_rays_z, 1);
    rs.cr_xy = d.dpitch_x;  // crystalSize.x / .y of the reference's kernels (init.py:736)
    rs.cr_z = d.dpitch_y;
    rs.w = h->d_w ? h->d_w + (meas_level ? h->n_meas[subset] : rs.proj0 * nbin) : nullptr;
    rs.mu = h->d_mu;
    return OMB_OK;
}

// First measurement (ray) of a subset in the all-subsets measurement order.
static int64_t subset_ray0(const omb_handle *h, const RaySet &rs, int32_t subset) {
    const bool meas_level = meas_level_subsets(h->desc);
    return meas_level ? h->n_meas[subset] : rs.proj0 * (int64_t)h->desc.n_rows_d * h->desc.n_cols_d;
}

static Frames one_frame_fp(const omb_handle *h, const float *img, float *y, int64_t m) {
    Frames f{};
    f.n = 1;
    f.img_in = img;
    f.img_stride = h->n_img;
    f.meas_out = y;
    f.meas_stride = m;
    return f;
}

static Frames one_frame_bp(const omb_handle *h, const float *y, float *img, int64_t m) {
    Frames f{};
    f.n = 1;
    f.meas = y;
    f.meas_stride = m;
    f.img = img;
    f.img_stride = h->n_img;
    return f;
}

// Ray-driven forward projection of a batch of frames (types 1 and 4).  With
// BF16 reads the images are first rounded into the handle's BF16 copies.
static int find_matrix(omb_handle *h, const RaySet &rs, const Orth *orth, cudaStream_t s, SysMat **out);

static int rays_forward(omb_handle *h, const RaySet &rs, const Frames &f_in, cudaStream_t s) {
    Frames f = f_in;
    if (h->read_mode == OMB_READ_BF16 && f.n > 0) {
        if (f.n > h->img16_frames)
            return set_error(OMB_ERR_INVALID, "more frames than omb_set_read_precision reserved BF16 copies for");
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = unet_to_bf16(f.img_in + fr * f.img_stride, h->d_img16 + fr * h->n_img, h->n_img, s);
            if (st != OMB_OK) return st;
        }
        f.img_in16 = h->d_img16;
        f.img_stride = h->n_img;
    }
    if ((h->desc.fp_type == 2 || h->desc.fp_type == 3) && h->desc.bp_type == h->desc.fp_type &&
        h->tune.siddon_bp_matrix && h->tof.nbins == 1 && !f.img_in16 && f.img_in && f.meas_out) {
        // the tube weights of the subset's system matrix (ray-major copy), built by its first call
        SysMat *sm = nullptr;
        const int fm = find_matrix(h, rs, &h->orth_bp, s, &sm);
        if (fm < 0) return fm;
        if (fm == OMB_OK && sm->rsent) return sysmat_forward(h->grid, *sm, f, rs.m_size, s);
    }
    if (h->desc.fp_type == 2 || h->desc.fp_type == 3) {
        if (f.img_in16) return set_error(OMB_ERR_UNSUPPORTED, "projector types 2 / 3 read FP32 images");
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = orth_forward(h->grid, rs, h->orth_fp, h->tof, h->desc.global_factor,
                                        f.img_in + fr * f.img_stride, f.meas_out + fr * f.meas_stride, s);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (h->desc.fp_type == 4) {
        if (rs.w || rs.mu) return set_error(OMB_ERR_UNSUPPORTED, "PET corrections are built for projector type 1");
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = interp_forward(h->grid, rs, h->tof, h->desc.global_factor, h->desc.dL,
                                          f.img_in16 ? nullptr : f.img_in + fr * f.img_stride,
                                          f.img_in16 ? f.img_in16 + fr * f.img_stride : nullptr,
                                          f.meas_out + fr * f.meas_stride, h->tune, s);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (rs.nr_xy * rs.nr_z > 1) {
        if (f.img_in16) return set_error(OMB_ERR_UNSUPPORTED, "multi-ray projection reads FP32 images");
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = multiray_forward(h->grid, rs, h->tof, h->desc.global_factor, f.img_in + fr * f.img_stride,
                                            f.meas_out + fr * f.meas_stride, h->tune.siddon_blocks_per_sm, s);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (!f.img_in16) attach_interleave(h, f, s);
    return siddon_forward(h->grid, rs, h->tof, h->desc.global_factor, f, h->tune, s);
}

// Ray-driven backprojection (float atomics, types 1 and 4) of a batch of
// frames into zeroed images; `sens` (zeroed) receives A^T 1 of the first
// frame's rays.  f.meas == NULL backprojects ones, f.img == NULL keeps only
// the sensitivity.
// Backprojection of f's frames through the subset's transposed system matrix (types 1-3, non-TOF), built
// by its first call; a build that does not fit in memory turns the matrix off for this handle and returns 1
// (the caller takes the ray-driven path).
static int find_matrix(omb_handle *h, const RaySet &rs, const Orth *orth, cudaStream_t s, SysMat **out) {
    *out = nullptr;
    for (auto &x : h->sysmats)
        if (x.proj0 == rs.proj0 && x.m_size == rs.m_size && x.cur_subset == rs.cur_subset) *out = &x;
    if (!*out) {
        SysMat nm;
        if (sysmat_build(h->grid, rs, h->desc.global_factor, nm, s, orth) != OMB_OK) {
            if (orth && std::string(omb_last_error()).find("not enough device memory") != std::string::npos) {
                h->tune.siddon_bp_matrix = 0;
                return 1;
            }
            return -1;
        }
        h->sysmats.push_back(nm);
        *out = &h->sysmats.back();
    }
    return OMB_OK;
}

static int matrix_backward(omb_handle *h, const RaySet &rs, const Frames &f, const Orth *orth, cudaStream_t s) {
    SysMat *sm = nullptr;
    const int fm = find_matrix(h, rs, orth, s, &sm);
    if (fm != OMB_OK) return fm;
    const int fb = f.n >= 8 ? 8 : (f.n >= 4 ? 4 : 1);
    if (fb > 1 && (int64_t)fb * rs.m_size > h->ym_floats) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
            return set_error(OMB_ERR_INVALID, "the system-matrix backprojection scratch grows on a call outside "
                                              "CUDA-graph capture (run one call first)");
        float *p = nullptr;
        if (cudaMalloc(&p, (size_t)fb * rs.m_size * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(OMB_ERR_CUDA, "allocating the system-matrix backprojection scratch failed");
        }
        if (h->d_ym) h->retired.push_back(h->d_ym);
        h->d_ym = p;
        h->ym_floats = (int64_t)fb * rs.m_size;
    }
    return sysmat_backward(h->grid, *sm, f, rs.m_size, h->d_ym, h->ym_floats, s);
}

static int rays_backward(omb_handle *h, const RaySet &rs, const Frames &f_in, float *sens, cudaStream_t s) {
    Frames f = f_in;
    if ((h->desc.bp_type == 2 || h->desc.bp_type == 3) && h->tune.siddon_bp_matrix && h->tof.nbins == 1 && !sens &&
        f.meas && f.img) {
        const int e = matrix_backward(h, rs, f, &h->orth_bp, s);
        if (e != 1) return e;
    }
    if (h->desc.bp_type == 2 || h->desc.bp_type == 3) {
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = orth_backward(h->grid, rs, h->orth_bp, h->tof, h->desc.global_factor,
                                         f.meas ? f.meas + fr * f.meas_stride : nullptr,
                                         f.img ? f.img + fr * f.img_stride : nullptr, fr == 0 ? sens : nullptr, s);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (h->desc.bp_type == 4) {
        if (rs.w || rs.mu) return set_error(OMB_ERR_UNSUPPORTED, "PET corrections are built for projector type 1");
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = interp_backward(h->grid, rs, h->tof, h->desc.global_factor, h->desc.dL,
                                           f.meas ? f.meas + fr * f.meas_stride : nullptr,
                                           f.img ? f.img + fr * f.img_stride : nullptr, fr == 0 ? sens : nullptr,
                                           nullptr, nullptr, h->tune, s);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (rs.nr_xy * rs.nr_z > 1) {
        for (int fr = 0; fr < f.n; ++fr) {
            const int st = multiray_backward(h->grid, rs, h->tof, h->desc.global_factor,
                                             f.meas ? f.meas + fr * f.meas_stride : nullptr,
                                             f.img ? f.img + fr * f.img_stride : nullptr, fr == 0 ? sens : nullptr,
                                             h->tune.siddon_blocks_per_sm, s);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (h->tune.siddon_bp_matrix && h->tof.nbins == 1 && !sens && f.meas && f.img) {
        // the subset's transposed system matrix, built by its first call
        return matrix_backward(h, rs, f, nullptr, s);
    }
    if (!sens && f.meas && f.img) attach_interleave(h, f, s);
    return siddon_backward(h->grid, rs, h->tof, h->desc.global_factor, f, sens, h->tune, s);
}

int omb::handle_subsets(const omb_handle *h) { return h ? h->desc.n_subsets : 0; }
Grid omb::handle_grid(const omb_handle *h) { return h ? h->grid : Grid{}; }
float omb::handle_epps(const omb_handle *h) { return h ? h->desc.epps : 0.f; }

int omb::sensitivity_raw(omb_handle *h, int32_t subset, float *sens, cudaStream_t s) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!sens) return set_error(OMB_ERR_INVALID, "sens pointer is NULL");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    if (h->desc.modality != OMB_PET_SINOGRAM || h->desc.bp_type < 1 || h->desc.bp_type > 4)
        return set_error(OMB_ERR_UNSUPPORTED, "omb_sensitivity needs a ray-driven PET backprojector (types 1 to 4)");
    // A^T 1 through the BP kernel's fused sensitivity accumulator, y = NULL.
    OMB_CUDA_TRY(cudaMemsetAsync(sens, 0, h->n_img * sizeof(float), s));
    return rays_backward(h, rs, one_frame_bp(h, nullptr, nullptr, rs.m_size), sens, s);
}

extern "C" {

int omb_abi_version(void) { return OMB_ABI_VERSION; }

const char *omb_last_error(void) { return g_last_error.c_str(); }

int omb_create(const omb_geometry_desc *desc, omb_handle **out) {
    if (!out) return set_error(OMB_ERR_INVALID, "output handle pointer is NULL");
    *out = nullptr;
    int st = validate(desc);
    if (st != OMB_OK) return st;
    omb_handle *h = new omb_handle();
    h->desc = *desc;
    h->desc.xy = nullptr;
    h->desc.z = nullptr;
    h->desc.tof_centers = nullptr;
    h->desc.n_meas = nullptr;
    h->n_meas.assign(desc->n_meas, desc->n_meas + desc->n_subsets + 1);
    cudaGetDevice(&h->device);
    Grid &g = h->grid;
    g.nx = (int)desc->nx; g.ny = (int)desc->ny; g.nz = (int)desc->nz;
    g.dx = desc->dx; g.dy = desc->dy; g.dz = desc->dz;
    g.bx = desc->bx; g.by = desc->by; g.bz = desc->bz;
    // bmax = b + N*d in float32, as the reference's host code forms it (projfunctions.py:397-399)
    g.mx = desc->bx + (float)desc->nx * desc->dx;
    g.my = desc->by + (float)desc->ny * desc->dy;
    g.mz = desc->bz + (float)desc->nz * desc->dz;
    h->n_img = (int64_t)desc->nx * desc->ny * desc->nz;
    Tof &t = h->tof;
    t.nbins = desc->tof_bins;
    t.epps = desc->epps;
    t.sigma_inv = desc->tof_bins > 1 ? 1.f / desc->sigma_x : 0.f;
    t.sigma_coef = 0.3989423f * t.sigma_inv;
    auto fail = [&](int code) {
        omb_destroy(h);
        return code;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&h->d_xy, desc->n_xy * sizeof(float))) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc xy"));
    if ((e = cudaMalloc(&h->d_z, (desc->n_z > 0 ? desc->n_z : 1) * sizeof(float))) != cudaSuccess)
        return fail(cuda_fail(e, "cudaMalloc z"));
    if ((e = cudaMemcpy(h->d_xy, desc->xy, desc->n_xy * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(cuda_fail(e, "upload xy"));
    if (desc->n_z > 0 && (e = cudaMemcpy(h->d_z, desc->z, desc->n_z * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(cuda_fail(e, "upload z"));
    h->desc.tr_index = nullptr;
    h->desc.ax_index = nullptr;
    if (desc->modality == OMB_PET_INDEXED) {
        const size_t nb = (size_t)desc->n_proj * 2 * sizeof(uint16_t);
        if ((e = cudaMalloc(&h->d_tr, nb)) != cudaSuccess || (e = cudaMalloc(&h->d_ax, nb)) != cudaSuccess)
            return fail(cuda_fail(e, "cudaMalloc event indices"));
        if ((e = cudaMemcpy(h->d_tr, desc->tr_index, nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(h->d_ax, desc->ax_index, nb, cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(cuda_fail(e, "upload event indices"));
    }
    if ((e = cudaMalloc(&h->d_tofc, kMaxTofBins * sizeof(float))) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc tof"));
    if ((e = cudaMemset(h->d_tofc, 0, kMaxTofBins * sizeof(float))) != cudaSuccess) return fail(cuda_fail(e, "clear tof"));
    if (desc->tof_bins > 1 &&
        (e = cudaMemcpy(h->d_tofc, desc->tof_centers, desc->tof_bins * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(cuda_fail(e, "upload tof centres"));
    t.centers = h->d_tofc;
    if (desc->fp_type == 5) {
        if ((e = cudaMalloc(&h->d_imgT, h->n_img * sizeof(float))) != cudaSuccess)
            return fail(cuda_fail(e, "cudaMalloc type-5 image copy"));
    }
    if (desc->bp_type == 5 || (desc->bp_type == 4 && desc->modality == OMB_CT_PANEL)) {
        std::vector<BddMap64> maps64;
        std::vector<BddProj> maps = bdd_maps(*desc, &maps64);
        if ((e = cudaMalloc(&h->d_bddp, maps.size() * sizeof(BddProj))) != cudaSuccess ||
            (e = cudaMalloc(&h->d_bddm64, maps64.size() * sizeof(BddMap64))) != cudaSuccess)
            return fail(cuda_fail(e, "cudaMalloc type-5 projection maps"));
        if ((e = cudaMemcpy(h->d_bddp, maps.data(), maps.size() * sizeof(BddProj), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(h->d_bddm64, maps64.data(), maps64.size() * sizeof(BddMap64), cudaMemcpyHostToDevice)) !=
                cudaSuccess)
            return fail(cuda_fail(e, "upload type-5 projection maps"));
    }
    if (desc->fixed64_workspace) {
        if ((e = cudaMalloc(&h->d_acc, 2 * h->n_img * sizeof(unsigned long long))) != cudaSuccess)
            return fail(cuda_fail(e, "cudaMalloc fixed-point accumulators"));
    }
    h->desc.vol_v = nullptr;
    if (desc->fp_type == 3 || desc->bp_type == 3) {
        if ((e = cudaMalloc(&h->d_vol, desc->n_vol_v * sizeof(float))) != cudaSuccess)
            return fail(cuda_fail(e, "cudaMalloc volume table"));
        if ((e = cudaMemcpy(h->d_vol, desc->vol_v, desc->n_vol_v * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(cuda_fail(e, "upload volume table"));
    }
    // the tube of each direction: the width argument follows the kernel's own type (init.py:650-655)
    auto tube = [&](int type) {
        Orth o{};
        o.type = type;
        o.width = type == 2 ? desc->tube_width : desc->tube_radius;
        o.xy = desc->orth_xy != 0;
        o.z = desc->orth_z != 0;
        o.bmin = desc->vol_bmin;
        o.bmax = desc->vol_bmax;
        o.vmax = desc->vol_vmax;
        o.v = h->d_vol;
        o.nv = type == 3 ? (int)desc->n_vol_v : 0;
        return o;
    };
    h->orth_fp = tube(desc->fp_type);
    h->orth_bp = tube(desc->bp_type);
    *out = h;
    return OMB_OK;
}

int omb_destroy(omb_handle *h) {
    if (!h) return OMB_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != h->device) cudaSetDevice(h->device);
    cudaFree(h->d_xy);
    cudaFree(h->d_tr);
    cudaFree(h->d_ax);
    cudaFree(h->d_z);
    cudaFree(h->d_tofc);
    cudaFree(h->d_acc);
    cudaFree(h->d_imgT);
    cudaFree(h->d_bddp);
    cudaFree(h->d_bddm64);
    cudaFree(h->d_img16);
    cudaFree(h->d_ilv);
    cudaFree(h->d_w);
    cudaFree(h->d_mu);
    cudaFree(h->d_rand);
    cudaFree(h->d_vol);
    for (auto &m : h->sysmats) sysmat_free(m);
    cudaFree(h->d_ym);
    for (void *p : h->retired) cudaFree(p);
    if (prev != h->device) cudaSetDevice(prev);
    delete h;
    return OMB_OK;
}

int64_t omb_measurement_count(const omb_handle *h, int32_t subset) {
    if (!h) return -1;
    RaySet rs{};
    if (ray_set(h, subset, rs) != OMB_OK) return -1;
    return rs.m_size * h->desc.tof_bins;
}

int64_t omb_image_count(const omb_handle *h) { return h ? h->n_img : -1; }

int omb_forward(omb_handle *h, int32_t subset, const float *image, float *y, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!image || !y) return set_error(OMB_ERR_INVALID, "image/y pointer is NULL");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    if (h->desc.fp_type == 5)
        return bdd_forward(h->grid, h->d_xy, h->d_z, rs.n_rows, rs.n_cols, rs.pitch_y, rs.proj0, rs.n_proj, image,
                           h->d_imgT, y, h->tune, (cudaStream_t)stream);
    return rays_forward(h, rs, one_frame_fp(h, image, y, rs.m_size), (cudaStream_t)stream);
}

int omb_forward_frames(omb_handle *h, int32_t subset, int32_t n_frames, const float *images, int64_t image_stride,
                       float *y, int64_t y_stride, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!images || !y) return set_error(OMB_ERR_INVALID, "images/y pointer is NULL");
    if (n_frames < 0) return set_error(OMB_ERR_INVALID, "n_frames must be >= 0");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    if (image_stride < h->n_img || y_stride < rs.m_size * h->desc.tof_bins)
        return set_error(OMB_ERR_INVALID, "frame strides smaller than one image / one measurement vector");
    if (h->desc.fp_type == 5) {
        for (int fr = 0; fr < n_frames; ++fr) {
            st = bdd_forward(h->grid, h->d_xy, h->d_z, rs.n_rows, rs.n_cols, rs.pitch_y, rs.proj0, rs.n_proj,
                             images + fr * image_stride, h->d_imgT, y + fr * y_stride, h->tune,
                             (cudaStream_t)stream);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    Frames f{};
    f.n = n_frames;
    f.img_in = images;
    f.img_stride = image_stride;
    f.meas_out = y;
    f.meas_stride = y_stride;
    return rays_forward(h, rs, f, (cudaStream_t)stream);
}

int omb_backward(omb_handle *h, int32_t subset, const float *y, float *image, float *sens, int32_t mode,
                 void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!image || !y) return set_error(OMB_ERR_INVALID, "image/y pointer is NULL");
    if (mode != OMB_BP_FLOAT_ATOMIC && mode != OMB_BP_FIXED64 && mode != OMB_BP_RAY)
        return set_error(OMB_ERR_INVALID, "unknown backprojection mode");
    if (mode == OMB_BP_FIXED64 && !h->d_acc)
        return set_error(OMB_ERR_INVALID, "fixed-point backprojection needs a handle created with fixed64_workspace");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nb = h->n_img * sizeof(float);
    if (h->desc.bp_type == 5) {
        if (mode == OMB_BP_FLOAT_ATOMIC)
            return bdd_backward(h->grid, h->d_bddp + rs.proj0, h->d_bddm64 + rs.proj0, rs.n_rows, rs.n_cols, rs.n_proj,
                                y, image, sens, h->tune, s);
        // ray-driven scatter: the exact adjoint of the forward projection
        if (mode == OMB_BP_FIXED64) {
            unsigned long long *acc = h->d_acc, *acc_s = sens ? h->d_acc + h->n_img : nullptr;
            OMB_CUDA_TRY(cudaMemsetAsync(h->d_acc, 0, (sens ? 2 : 1) * h->n_img * sizeof(unsigned long long), s));
            st = bdd_backward_ray(h->grid, rs.xy, rs.z, rs.n_rows, rs.n_cols, rs.pitch_y, rs.proj0, rs.n_proj, y,
                                  nullptr, nullptr, acc, acc_s, s);
            if (st != OMB_OK) return st;
            st = fixed_to_float(acc, image, h->n_img, s);
            if (st == OMB_OK && sens) st = fixed_to_float(acc_s, sens, h->n_img, s);
            return st;
        }
        OMB_CUDA_TRY(cudaMemsetAsync(image, 0, nb, s));
        if (sens) OMB_CUDA_TRY(cudaMemsetAsync(sens, 0, nb, s));
        return bdd_backward_ray(h->grid, rs.xy, rs.z, rs.n_rows, rs.n_cols, rs.pitch_y, rs.proj0, rs.n_proj, y, image,
                                sens, nullptr, nullptr, s);
    }
    if (h->desc.bp_type == 4 && h->desc.modality == OMB_CT_PANEL) {
        if (mode != OMB_BP_FLOAT_ATOMIC)
            return set_error(OMB_ERR_UNSUPPORTED, "the type-4 CT backprojection is a gather; it has no fixed-point "
                                                  "or ray-driven mode");
        return interp_ct_backward(h->grid, h->d_bddp + rs.proj0, rs.n_rows, rs.n_cols, rs.n_proj, h->desc.kerroin, y,
                                  image, sens, s);
    }
    if (mode == OMB_BP_FIXED64) {
        if (rs.nr_xy * rs.nr_z > 1)
            return set_error(OMB_ERR_UNSUPPORTED, "the fixed-point backprojection takes one ray per LOR");
        unsigned long long *acc = h->d_acc, *acc_s = sens ? h->d_acc + h->n_img : nullptr;
        OMB_CUDA_TRY(cudaMemsetAsync(h->d_acc, 0, (sens ? 2 : 1) * h->n_img * sizeof(unsigned long long), s));
        if (h->desc.bp_type == 4)
            st = interp_backward(h->grid, rs, h->tof, h->desc.global_factor, h->desc.dL, y, nullptr, nullptr, acc,
                                 acc_s, h->tune, s);
        else
            st = siddon_backward_fixed(h->grid, rs, h->tof, h->desc.global_factor, y, acc, acc_s, s);
        if (st != OMB_OK) return st;
        st = fixed_to_float(acc, image, h->n_img, s);
        if (st == OMB_OK && sens) st = fixed_to_float(acc_s, sens, h->n_img, s);
        return st;
    }
    OMB_CUDA_TRY(cudaMemsetAsync(image, 0, nb, s));
    if (sens) OMB_CUDA_TRY(cudaMemsetAsync(sens, 0, nb, s));
    return rays_backward(h, rs, one_frame_bp(h, y, image, rs.m_size), sens, s);
}

int omb_backward_frames(omb_handle *h, int32_t subset, int32_t n_frames, const float *y, int64_t y_stride,
                        float *images, int64_t image_stride, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!images || !y) return set_error(OMB_ERR_INVALID, "images/y pointer is NULL");
    if (n_frames < 0) return set_error(OMB_ERR_INVALID, "n_frames must be >= 0");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    if (image_stride < h->n_img || y_stride < rs.m_size * h->desc.tof_bins)
        return set_error(OMB_ERR_INVALID, "frame strides smaller than one image / one measurement vector");
    cudaStream_t s = (cudaStream_t)stream;
    if (h->desc.bp_type == 5 || (h->desc.bp_type == 4 && h->desc.modality == OMB_CT_PANEL)) {
        for (int fr = 0; fr < n_frames; ++fr) {
            st = omb_backward(h, subset, y + fr * y_stride, images + fr * image_stride, nullptr, OMB_BP_FLOAT_ATOMIC,
                              stream);
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    if (image_stride == h->n_img) {
        OMB_CUDA_TRY(cudaMemsetAsync(images, 0, (size_t)n_frames * h->n_img * sizeof(float), s));
    } else {
        OMB_CUDA_TRY(cudaMemset2DAsync(images, image_stride * sizeof(float), 0, h->n_img * sizeof(float), n_frames, s));
    }
    Frames f{};
    f.n = n_frames;
    f.meas = y;
    f.meas_stride = y_stride;
    f.img = images;
    f.img_stride = image_stride;
    return rays_backward(h, rs, f, nullptr, s);
}

int omb_sensitivity(omb_handle *h, int32_t subset, float *sens, void *stream) {
    const int st = sensitivity_raw(h, subset, sens, (cudaStream_t)stream);
    if (st != OMB_OK) return st;
    return clamp_min(sens, h->n_img, h->desc.epps, (cudaStream_t)stream);
}

int omb_osem_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const float *sens,
                    float *work_meas, float *work_img, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!image || !y_subset || !sens || !work_meas || !work_img)
        return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_osem_subset");
    if (h->desc.modality == OMB_CT_PANEL) return set_error(OMB_ERR_UNSUPPORTED, "OSEM sub-iteration is PET-only");
    if (h->desc.fp_type < 1 || h->desc.fp_type > 4 || h->desc.bp_type < 1 || h->desc.bp_type > 4)
        return set_error(OMB_ERR_UNSUPPORTED, "omb_osem_subset needs projector types 1 to 4");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const float eps = h->desc.epps;
    const int64_t m = rs.m_size * h->desc.tof_bins;
    st = rays_forward(h, rs, one_frame_fp(h, image, work_meas, rs.m_size), s);
    if (st != OMB_OK) return st;
    if (h->d_rand)
        st = osem_ratio_randoms(y_subset, m, work_meas, m, m, 1, h->d_rand + subset_ray0(h, rs, subset), rs.m_size,
                                eps, s);
    else
        st = osem_ratio(y_subset, work_meas, m, eps, s);
    if (st != OMB_OK) return st;
    OMB_CUDA_TRY(cudaMemsetAsync(work_img, 0, h->n_img * sizeof(float), s));
    st = rays_backward(h, rs, one_frame_bp(h, work_meas, work_img, rs.m_size), nullptr, s);
    if (st != OMB_OK) return st;
    return em_update(image, sens, work_img, h->n_img, eps, s);
}

int omb_osl_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const float *sens,
                   const float *du, float *work_meas, float *work_img, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!image || !y_subset || !sens || !du || !work_meas || !work_img)
        return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_osl_subset");
    if (h->desc.modality == OMB_CT_PANEL) return set_error(OMB_ERR_UNSUPPORTED, "OSEM sub-iteration is PET-only");
    if (h->desc.fp_type < 1 || h->desc.fp_type > 4 || h->desc.bp_type < 1 || h->desc.bp_type > 4)
        return set_error(OMB_ERR_UNSUPPORTED, "omb_osl_subset needs projector types 1 to 4");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const float eps = h->desc.epps;
    const int64_t m = rs.m_size * h->desc.tof_bins;
    st = rays_forward(h, rs, one_frame_fp(h, image, work_meas, rs.m_size), s);
    if (st != OMB_OK) return st;
    if (h->d_rand)
        st = osem_ratio_randoms(y_subset, m, work_meas, m, m, 1, h->d_rand + subset_ray0(h, rs, subset), rs.m_size,
                                eps, s);
    else
        st = osem_ratio(y_subset, work_meas, m, eps, s);
    if (st != OMB_OK) return st;
    OMB_CUDA_TRY(cudaMemsetAsync(work_img, 0, h->n_img * sizeof(float), s));
    st = rays_backward(h, rs, one_frame_bp(h, work_meas, work_img, rs.m_size), nullptr, s);
    if (st != OMB_OK) return st;
    return osl_update(image, sens, du, work_img, h->n_img, s);
}

}  // extern "C"

namespace omb {
int relaxed_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const RelaxedArgs &a,
                   float *work_meas, float *work_img, cudaStream_t s) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!image || !y_subset || (a.kind == kRosem && !a.sens) || !work_meas || !work_img)
        return set_error(OMB_ERR_INVALID, "NULL buffer passed to a relaxed sub-iteration");
    if (a.precond < 0 || a.precond > 2 || (a.precond && !a.precond_d))
        return set_error(OMB_ERR_INVALID, "image preconditioner: mode 0..2, modes 1 and 2 need their D image");
    if (h->desc.modality == OMB_CT_PANEL)
        return set_error(OMB_ERR_UNSUPPORTED, "the relaxed sub-iterations are PET-only");
    if (h->desc.fp_type < 1 || h->desc.fp_type > 4 || h->desc.bp_type < 1 || h->desc.bp_type > 4)
        return set_error(OMB_ERR_UNSUPPORTED, "the relaxed sub-iterations need projector types 1 to 4");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    const float eps = h->desc.epps;
    const int64_t m = rs.m_size * h->desc.tof_bins;
    st = rays_forward(h, rs, one_frame_fp(h, image, work_meas, rs.m_size), s);
    if (st != OMB_OK) return st;
    // ROSEM: y / fp; RAMLA, BSREM, MRAMLA, MBSREM: y / fp - 1; PKMA: 1 - y / fp
    // (computeForwardProject.h:76-101, 98-122, 126-150, 153-180)
    const float shift = a.kind == kRosem ? 0.f : 1.f;
    const float sign = a.kind == kPkma ? -1.f : 1.f;
    st = ratio_shift(y_subset, work_meas, m, h->d_rand ? h->d_rand + subset_ray0(h, rs, subset) : nullptr,
                     rs.m_size, eps, shift, sign, s);
    if (st != OMB_OK) return st;
    // measurement preconditioner type 0: the ratio over A 1 (computeForwardProject.h:149, 183;
    // functions.hpp:2156-2166)
    if (a.meas_m && (st = div_inplace(work_meas, a.meas_m, m, s)) != OMB_OK) return st;
    OMB_CUDA_TRY(cudaMemsetAsync(work_img, 0, h->n_img * sizeof(float), s));
    st = rays_backward(h, rs, one_frame_bp(h, work_meas, work_img, rs.m_size), nullptr, s);
    if (st != OMB_OK) return st;
    if ((a.kind == kPkma || a.kind == kMbsrem) && (a.ext_on || a.auto_relax || a.relax_scaling)) {
        // the gradient preconditioned in place, then (PKMA) the relaxation from the norms
        PrecondExt p = a.ext;
        p.fold = a.kind == kMbsrem ? 1 : 0;
        p.upper = a.upper;
        if (p.gradF && (st = precond_gradient(image, a.gradF, h->grid, p, a.work, s)) != OMB_OK) return st;
        if ((st = precond_apply(work_img, a.du, image, h->n_img, p, s)) != OMB_OK) return st;
        if (p.filt_h) {
            // type 5 last (functions.hpp:2093-2099), in the filtering sub-iterations only
            FilterGate gt;
            gt.it = p.it;
            gt.n_sub = p.n_sub;
            gt.sub = p.sub;
            gt.K = p.filt_K;
            if (!p.filt_tmp || !p.it) return set_error(OMB_ERR_INVALID, "the image filter needs its scratch and counter");
            if ((st = image_filter(work_img, p.filt_tmp, h->grid.nx, h->grid.ny, h->grid.nz, p.filt_h, p.filt_nf, gt, s)) !=
                OMB_OK)
                return st;
        }
        if (a.kind == kPkma && (a.auto_relax || a.relax_scaling)) {
            if (!a.lam.lam || !a.lam.iter || !a.work)
                return set_error(OMB_ERR_INVALID, "PKMA relaxation needs the device schedule and workspace");
            double *w1 = a.work + precond_workspace_bytes() / sizeof(double);
            double *w2 = w1 + dot_workspace_bytes() / sizeof(double);
            const size_t off = dot_workspace_bytes() / sizeof(double) - 2;
            if ((st = dot2(image, work_img, h->n_img, w1, s)) != OMB_OK) return st;  // x.g, g.g
            if ((st = dot2(work_img, image, h->n_img, w2, s)) != OMB_OK) return st;  // g.x, x.x
            if ((st = pkma_relax(const_cast<float *>(a.lam.lam), a.lam.iter, p.sub, w1 + off, w2 + off,
                                 a.auto_relax, a.relax_scaling, s)) != OMB_OK)
                return st;
        }
        if (a.kind == kPkma)
            return pkma_update(image, work_img, nullptr, h->n_img, a.lam, a.alpha, eps, a.positivity, nullptr, 0, s);
        return mbsrem_update(image, work_img, nullptr, h->n_img, a.lam, eps, a.upper, a.positivity, nullptr, 0, s);
    }
    switch (a.kind) {
        case kRosem: return rosem_update(image, a.sens, work_img, h->n_img, a.lam, s);
        case kRamla: return bsrem_update(image, work_img, h->n_img, a.lam, eps, a.positivity, s);
        case kPkma:
            return pkma_update(image, work_img, a.du, h->n_img, a.lam, a.alpha, eps, a.positivity, a.precond_d,
                               a.precond, s);
        case kMbsrem:
            return mbsrem_update(image, work_img, a.du, h->n_img, a.lam, eps, a.upper, a.positivity, a.precond_d,
                                 a.precond, s);
        default: return set_error(OMB_ERR_INVALID, "unknown relaxed update");
    }
}
}  // namespace omb

extern "C" {

int omb_rosem_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, const float *sens,
                     float lambda, float *work_meas, float *work_img, void *stream) {
    RelaxedArgs a;
    a.kind = kRosem;
    a.sens = sens;
    a.lam.v = lambda;
    return relaxed_subset(h, subset, image, y_subset, a, work_meas, work_img, (cudaStream_t)stream);
}

int omb_ramla_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, float lambda,
                     int32_t positivity, float *work_meas, float *work_img, void *stream) {
    RelaxedArgs a;
    a.kind = kRamla;
    a.lam.v = lambda;
    a.positivity = positivity != 0;
    return relaxed_subset(h, subset, image, y_subset, a, work_meas, work_img, (cudaStream_t)stream);
}

int omb_pkma_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, float lambda, float alpha,
                    const float *du, int32_t positivity, const float *precond_d, int32_t precond, float *work_meas,
                    float *work_img, void *stream) {
    RelaxedArgs a;
    a.precond_d = precond_d;
    a.precond = precond;
    a.kind = kPkma;
    a.du = du;
    a.lam.v = lambda;
    a.alpha.v = alpha;
    a.positivity = positivity != 0;
    return relaxed_subset(h, subset, image, y_subset, a, work_meas, work_img, (cudaStream_t)stream);
}

int omb_mbsrem_subset(omb_handle *h, int32_t subset, float *image, const float *y_subset, float lambda,
                      float upper, const float *du, int32_t positivity, const float *precond_d, int32_t precond,
                      float *work_meas, float *work_img, void *stream) {
    if (!(upper > 0.f)) return set_error(OMB_ERR_INVALID, "the upper bound U must be positive");
    RelaxedArgs a;
    a.precond_d = precond_d;
    a.precond = precond;
    a.kind = kMbsrem;
    a.du = du;
    a.lam.v = lambda;
    a.upper = upper;
    a.positivity = positivity != 0;
    return relaxed_subset(h, subset, image, y_subset, a, work_meas, work_img, (cudaStream_t)stream);
}

int omb_map_step(float *image, const float *du, int64_t n, float lambda, float epps, void *stream) {
    if (n < 0) return set_error(OMB_ERR_INVALID, "n must be >= 0");
    if (n > 0 && (!image || !du)) return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_map_step");
    Relax lam;
    lam.v = lambda;
    return map_step(image, du, n, lam, epps, (cudaStream_t)stream);
}

int omb_osem_subset_frames(omb_handle *h, int32_t subset, int32_t n_frames, float *images, int64_t image_stride,
                           const float *y_subset, int64_t y_stride, const float *sens, float *work_meas,
                           float *work_img, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!images || !y_subset || !sens || !work_meas || !work_img)
        return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_osem_subset_frames");
    if (n_frames < 0) return set_error(OMB_ERR_INVALID, "n_frames must be >= 0");
    if (h->desc.modality == OMB_CT_PANEL) return set_error(OMB_ERR_UNSUPPORTED, "OSEM sub-iteration is PET-only");
    if (h->desc.fp_type < 1 || h->desc.fp_type > 4 || h->desc.bp_type < 1 || h->desc.bp_type > 4)
        return set_error(OMB_ERR_UNSUPPORTED, "omb_osem_subset_frames needs projector types 1 to 4");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    const int64_t m = rs.m_size * h->desc.tof_bins;
    if (image_stride < h->n_img || y_stride < m)
        return set_error(OMB_ERR_INVALID, "frame strides smaller than one image / one measurement vector");
    if (n_frames == 0) return OMB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const float eps = h->desc.epps;
    Frames f{};
    f.n = n_frames;
    f.img_in = images;
    f.img_stride = image_stride;
    f.meas_out = work_meas;
    f.meas_stride = m;
    st = rays_forward(h, rs, f, s);
    if (st != OMB_OK) return st;
    if (h->d_rand)
        st = osem_ratio_randoms(y_subset, y_stride, work_meas, m, m, n_frames, h->d_rand + subset_ray0(h, rs, subset),
                                rs.m_size, eps, s);
    else
        st = osem_ratio_frames(y_subset, y_stride, work_meas, m, m, n_frames, eps, s);
    if (st != OMB_OK) return st;
    OMB_CUDA_TRY(cudaMemsetAsync(work_img, 0, (size_t)n_frames * h->n_img * sizeof(float), s));
    Frames b{};
    b.n = n_frames;
    b.meas = work_meas;
    b.meas_stride = m;
    b.img = work_img;
    b.img_stride = h->n_img;
    st = rays_backward(h, rs, b, nullptr, s);
    if (st != OMB_OK) return st;
    return em_update_frames(images, image_stride, sens, work_img, h->n_img, h->n_img, n_frames, eps, s);
}

int omb_system_matrix_nnz(omb_handle *h, int32_t subset, int64_t *out_host) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!out_host) return set_error(OMB_ERR_INVALID, "output pointer is NULL");
    RaySet rs{};
    const int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    *out_host = 0;
    for (const auto &x : h->sysmats)
        if (x.proj0 == rs.proj0 && x.m_size == rs.m_size && x.cur_subset == rs.cur_subset) *out_host = x.nnz;
    return OMB_OK;
}

int omb_intersection_count(omb_handle *h, int32_t subset, int64_t *out_host, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!out_host) return set_error(OMB_ERR_INVALID, "output pointer is NULL");
    if (h->desc.fp_type != 1) return set_error(OMB_ERR_UNSUPPORTED, "intersection counts are for projector type 1");
    RaySet rs{};
    int st = ray_set(h, subset, rs);
    if (st != OMB_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long *d = nullptr;
    OMB_CUDA_TRY(cudaMallocAsync(&d, sizeof(unsigned long long), s));
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) st = siddon_count(h->grid, rs, h->tof, d, s);
    unsigned long long v = 0;
    if (e == cudaSuccess && st == OMB_OK) e = cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "intersection count");
    if (st != OMB_OK) return st;
    *out_host = (int64_t)v;
    return OMB_OK;
}

// ---------------------------------------------------------------------------
// Launch-shape tuning
// ---------------------------------------------------------------------------

static bool one_of(int v, std::initializer_list<int> ok) {
    for (int o : ok)
        if (v == o) return true;
    return false;
}

static int tuning_from(const omb_tuning *in, Tuning &t) {
    if (!in) return set_error(OMB_ERR_INVALID, "tuning pointer is NULL");
    if (in->struct_size != sizeof(omb_tuning))
        return set_error(OMB_ERR_INVALID, "omb_tuning.struct_size does not match this library (" +
                                              std::to_string(sizeof(omb_tuning)) + " bytes)");
    if (in->siddon_blocks_per_sm < 1 || in->siddon_blocks_per_sm > 32)
        return set_error(OMB_ERR_INVALID, "siddon_blocks_per_sm must be in 1..32");
    if (!one_of(in->siddon_frames_per_walk, {1, 2, 4, 8}))
        return set_error(OMB_ERR_INVALID, "siddon_frames_per_walk must be 1, 2, 4 or 8");
    if (!one_of(in->bdd_fp_columns, {8, 16})) return set_error(OMB_ERR_INVALID, "bdd_fp_columns must be 8 or 16");
    if (!one_of(in->bdd_bp_zrun, {4, 8, 16})) return set_error(OMB_ERR_INVALID, "bdd_bp_zrun must be 4, 8 or 16");
    if (!one_of(in->bdd_fp_block_rows, {4, 8}) || !one_of(in->bdd_bp_block_rows, {4, 8}))
        return set_error(OMB_ERR_INVALID, "bdd block rows must be 4 or 8");
    if (!one_of(in->siddon_frame_layout, {0, 1})) return set_error(OMB_ERR_INVALID, "siddon_frame_layout must be 0 or 1");
    if (!one_of(in->siddon_fp_steps, {1, 2, 4})) return set_error(OMB_ERR_INVALID, "siddon_fp_steps must be 1, 2 or 4");
    if (!one_of(in->bdd_fp_staged, {0, 1}) || !one_of(in->bdd_bp_staged, {0, 1}))
        return set_error(OMB_ERR_INVALID, "bdd_fp_staged and bdd_bp_staged must be 0 or 1");
    if (!one_of(in->siddon_bp_matrix, {0, 1})) return set_error(OMB_ERR_INVALID, "siddon_bp_matrix must be 0 or 1");
    t.siddon_blocks_per_sm = in->siddon_blocks_per_sm;
    t.siddon_frames = in->siddon_frames_per_walk;
    t.bdd_fp_cols = in->bdd_fp_columns;
    t.bdd_bp_z = in->bdd_bp_zrun;
    t.bdd_fp_rows = in->bdd_fp_block_rows;
    t.bdd_bp_rows = in->bdd_bp_block_rows;
    t.siddon_layout = in->siddon_frame_layout;
    t.siddon_fp_steps = in->siddon_fp_steps;
    t.bdd_fp_staged = in->bdd_fp_staged;
    t.bdd_bp_staged = in->bdd_bp_staged;
    t.siddon_bp_matrix = in->siddon_bp_matrix;
    return OMB_OK;
}

static void tuning_to(const Tuning &t, omb_tuning *out) {
    out->struct_size = sizeof(omb_tuning);
    out->siddon_blocks_per_sm = t.siddon_blocks_per_sm;
    out->siddon_frames_per_walk = t.siddon_frames;
    out->bdd_fp_columns = t.bdd_fp_cols;
    out->bdd_bp_zrun = t.bdd_bp_z;
    out->bdd_fp_block_rows = t.bdd_fp_rows;
    out->bdd_bp_block_rows = t.bdd_bp_rows;
    out->siddon_frame_layout = t.siddon_layout;
    out->siddon_fp_steps = t.siddon_fp_steps;
    out->bdd_fp_staged = t.bdd_fp_staged;
    out->bdd_bp_staged = t.bdd_bp_staged;
    out->siddon_bp_matrix = t.siddon_bp_matrix;
}

int omb_set_corrections(omb_handle *h, const float *meas_weights, int64_t n_weights, const float *atten_image,
                        int64_t n_atten, void *stream) {
    // the system matrices fold the corrections into their weights (retired,
    // not freed: a captured graph may still address them)
    if (h) {
        for (auto &m : h->sysmats) {
            h->retired.push_back(m.off);
            h->retired.push_back(m.ent);
            h->retired.push_back(m.soff);
            h->retired.push_back(m.sent);
            h->retired.push_back(m.rsoff);
            h->retired.push_back(m.rsent);
            h->retired.push_back(m.rcnt);
        }
        h->sysmats.clear();
    }
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if ((meas_weights || atten_image) && h->desc.modality == OMB_CT_PANEL)
        return set_error(OMB_ERR_UNSUPPORTED, "corrections apply to PET data");
    // rays of all subsets (TOF bins share their ray's weight)
    const bool meas_level = meas_level_subsets(h->desc);
    const int64_t total = meas_level ? h->n_meas[h->desc.n_subsets]
                                     : h->desc.n_proj * (int64_t)h->desc.n_rows_d * h->desc.n_cols_d;
    if (meas_weights && n_weights != total)
        return set_error(OMB_ERR_INVALID, "meas_weights must hold one value per measurement of all subsets (" +
                                              std::to_string(total) + ")");
    if (atten_image && n_atten != h->n_img)
        return set_error(OMB_ERR_INVALID, "atten_image must hold one value per voxel");
    cudaStream_t s = (cudaStream_t)stream;
    auto replace = [&](float *&dst, const float *src, int64_t n) -> int {
        if (dst) h->retired.push_back(dst);  // a captured graph may still read it
        dst = nullptr;
        if (!src) return OMB_OK;
        OMB_CUDA_TRY(cudaMalloc(&dst, (size_t)n * sizeof(float)));
        OMB_CUDA_TRY(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(float), cudaMemcpyDefault, s));
        OMB_CUDA_TRY(cudaStreamSynchronize(s));
        return OMB_OK;
    };
    int st = replace(h->d_w, meas_weights, n_weights);
    if (st == OMB_OK) st = replace(h->d_mu, atten_image, n_atten);
    return st;
}

int omb_set_randoms(omb_handle *h, const float *randoms, int64_t n, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (randoms && h->desc.modality == OMB_CT_PANEL) return set_error(OMB_ERR_UNSUPPORTED, "randoms apply to PET data");
    const bool meas_level = meas_level_subsets(h->desc);
    const int64_t total = meas_level ? h->n_meas[h->desc.n_subsets]
                                     : h->desc.n_proj * (int64_t)h->desc.n_rows_d * h->desc.n_cols_d;
    if (randoms && n != total)
        return set_error(OMB_ERR_INVALID, "randoms must hold one value per measurement of all subsets (" +
                                              std::to_string(total) + ")");
    if (h->d_rand) h->retired.push_back(h->d_rand);
    h->d_rand = nullptr;
    if (!randoms) return OMB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    OMB_CUDA_TRY(cudaMalloc(&h->d_rand, (size_t)n * sizeof(float)));
    OMB_CUDA_TRY(cudaMemcpyAsync(h->d_rand, randoms, (size_t)n * sizeof(float), cudaMemcpyDefault, s));
    OMB_CUDA_TRY(cudaStreamSynchronize(s));
    return OMB_OK;
}

int omb_take_device_error(void) {
    const int v = take_device_error();
    if (v < 0) return set_error(OMB_ERR_CUDA, "reading the device error word failed");
    return v;
}

int omb_get_tuning(const omb_handle *h, omb_tuning *out) {
    if (!h || !out) return set_error(OMB_ERR_INVALID, "handle/output pointer is NULL");
    if (out->struct_size != sizeof(omb_tuning))
        return set_error(OMB_ERR_INVALID, "omb_tuning.struct_size does not match this library");
    tuning_to(h->tune, out);
    return OMB_OK;
}

int omb_set_tuning(omb_handle *h, const omb_tuning *in) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    Tuning t{};
    int st = tuning_from(in, t);
    if (st == OMB_OK) h->tune = t;
    return st;
}

int omb_set_read_precision(omb_handle *h, int32_t mode, int32_t max_frames) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (mode != OMB_READ_FP32 && mode != OMB_READ_BF16) return set_error(OMB_ERR_INVALID, "unknown read precision");
    if (mode == OMB_READ_BF16 && h->desc.fp_type != 1 && h->desc.fp_type != 4)
        return set_error(OMB_ERR_UNSUPPORTED, "BF16 image reads are built for forward projector types 1 and 4");
    if (mode == OMB_READ_BF16 && max_frames < 1) return set_error(OMB_ERR_INVALID, "max_frames must be >= 1");
    if (mode == OMB_READ_BF16 && max_frames > h->img16_frames) {
        __nv_bfloat16 *p = nullptr;
        const cudaError_t e = cudaMalloc(&p, (size_t)max_frames * h->n_img * sizeof(__nv_bfloat16));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc BF16 image copies");
        if (h->d_img16) h->retired.push_back(h->d_img16);
        h->d_img16 = p;
        h->img16_frames = max_frames;
    }
    h->read_mode = mode;
    return OMB_OK;
}

int omb_autotune(omb_handle *h, int32_t n_frames, int32_t repeats, omb_tuning *out, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (n_frames < 1 || repeats < 1) return set_error(OMB_ERR_INVALID, "n_frames and repeats must be >= 1");
    if (out && out->struct_size != sizeof(omb_tuning))
        return set_error(OMB_ERR_INVALID, "omb_tuning.struct_size does not match this library");
    // ray-driven kernels (types 1 and 4 forward, PET types 1 and 4 backward)
    // share the blocks-per-SM and frames-per-walk shapes
    const bool ray_fp = h->desc.fp_type == 1 || h->desc.fp_type == 4;
    const bool ray_bp = h->desc.bp_type == 1 || (h->desc.bp_type == 4 && h->desc.modality != OMB_CT_PANEL);
    const bool siddon = ray_fp || ray_bp;
    if (!(h->desc.fp_type == 1 && h->desc.bp_type == 1) || h->desc.tof_bins > 1) n_frames = 1;
    const int64_t m = omb_measurement_count(h, -1);
    if (m < 0) return -1;
    const int64_t n = h->n_img;
    cudaStream_t s = (cudaStream_t)stream;
    float *img = nullptr, *y = nullptr, *back = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = OMB_OK;
    cudaError_t e = cudaMallocAsync(&img, (size_t)n_frames * n * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&back, (size_t)n_frames * n * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&y, (size_t)n_frames * m * sizeof(float), s);
    // positive filler (byte 0x3C -> 0.0115f): timing does not depend on values
    if (e == cudaSuccess) e = cudaMemsetAsync(img, 0x3C, (size_t)n_frames * n * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(y, 0x3C, (size_t)n_frames * m * sizeof(float), s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const Tuning saved = h->tune;
    auto fwd = [&]() { return omb_forward_frames(h, -1, n_frames, img, n, y, m, stream); };
    auto bwd = [&]() { return omb_backward_frames(h, -1, n_frames, y, m, back, n, stream); };
    // mean milliseconds of `repeats` calls of f after one warm-up call; < 0 on failure
    auto timed = [&](auto &&f) -> float {
        if (f() != OMB_OK) return -1.f;
        if (cudaEventRecord(e0, s) != cudaSuccess) return -1.f;
        for (int r = 0; r < repeats; ++r)
            if (f() != OMB_OK) return -1.f;
        float ms = -1.f;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            return -1.f;
        return ms / repeats;
    };
    Tuning best = saved;
    if (e == cudaSuccess && siddon) {
        float best_ms = 3.4e38f;
        const int frames_max = h->desc.tof_bins > 1 ? 1 : 8;
        for (int ps : {2, 4, 8, 16}) {
            for (int fr = 1; fr <= frames_max && fr <= n_frames && st == OMB_OK; fr *= 2) {
                // the voxel-interleaved layout applies to type-1 walks of 4 or 8 frames
                const bool both = fr >= 4 && h->desc.fp_type == 1 && h->desc.bp_type == 1;
                for (int layout = both ? 0 : saved.siddon_layout; layout <= (both ? 1 : saved.siddon_layout);
                     ++layout) {
                    h->tune = saved;
                    h->tune.siddon_blocks_per_sm = ps;
                    h->tune.siddon_frames = fr;
                    h->tune.siddon_layout = layout;
                    const float a = ray_fp ? timed(fwd) : 0.f, b = a < 0.f ? -1.f : (ray_bp ? timed(bwd) : 0.f);
                    if (a < 0.f || b < 0.f) {
                        st = -1;
                        break;
                    }
                    if (a + b < best_ms) {
                        best_ms = a + b;
                        best.siddon_blocks_per_sm = ps;
                        best.siddon_frames = fr;
                        best.siddon_layout = layout;
                    }
                }
            }
        }
    }
    // then the forward walk's batched crossings (type 1 without TOF)
    if (e == cudaSuccess && st == OMB_OK && h->desc.fp_type == 1 && h->desc.tof_bins == 1) {
        float best_ms = 3.4e38f;
        for (int k : {1, 2, 4}) {
            h->tune = best;
            h->tune.siddon_fp_steps = k;
            const float a = timed(fwd);
            if (a < 0.f) {
                st = -1;
                break;
            }
            if (a < best_ms) {
                best_ms = a;
                best.siddon_fp_steps = k;
            }
        }
    }
    // then the type-1 non-TOF backprojection through the resident transposed
    // system matrix, when its 8 bytes a crossing fit in half the free memory
    if (e == cudaSuccess && st == OMB_OK && h->desc.bp_type == 1 && h->desc.tof_bins == 1 &&
        h->desc.n_rays_xy * h->desc.n_rays_z <= 1) {
        int64_t crossings = 0;
        size_t free_b = 0, total_b = 0;
        if (omb_intersection_count(h, -1, &crossings, stream) == OMB_OK && cudaStreamSynchronize(s) == cudaSuccess &&
            cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
            (double)crossings * 8.0 + 8.0 * (double)m * 4.0 < 0.5 * (double)free_b) {
            h->tune = best;
            h->tune.siddon_bp_matrix = 0;
            const float b0 = timed(bwd);
            h->tune.siddon_bp_matrix = 1;
            const float b1 = timed(bwd);
            if (b0 < 0.f || b1 < 0.f) st = -1;
            else best.siddon_bp_matrix = b1 < b0 ? 1 : 0;
            if (!best.siddon_bp_matrix) {
                for (auto &x : h->sysmats) sysmat_free(x);
                h->sysmats.clear();
            }
        } else {
            cudaGetLastError();
        }
    }
    // types 2 / 3 (non-TOF): the tube weights through the transposed system matrix when it fits and is faster
    // (a build that does not fit turns the matrix off again)
    if (e == cudaSuccess && st == OMB_OK && (h->desc.bp_type == 2 || h->desc.bp_type == 3) && h->desc.tof_bins == 1) {
        h->tune = best;
        h->tune.siddon_bp_matrix = 0;
        const float b0 = timed(bwd);
        h->tune.siddon_bp_matrix = 1;
        const float b1 = timed(bwd);
        if (b0 < 0.f || b1 < 0.f) st = -1;
        else best.siddon_bp_matrix = h->tune.siddon_bp_matrix && b1 < b0 ? 1 : 0;
        if (!best.siddon_bp_matrix) {
            for (auto &x : h->sysmats) sysmat_free(x);
            h->sysmats.clear();
        }
    }
    if (e == cudaSuccess && st == OMB_OK && h->desc.fp_type == 5) {
        float best_ms = 3.4e38f;
        // (columns, warps per block, staged); the staged kernel has 8 or 16 columns per thread, 32 per CTA
        const int shapes[6][3] = {{8, 4, 0}, {8, 8, 0}, {16, 4, 0}, {16, 8, 0}, {8, 4, 1}, {16, 4, 1}};
        for (const auto &sh : shapes) {
            h->tune = best;
            h->tune.bdd_fp_cols = sh[0];
            h->tune.bdd_fp_rows = sh[1];
            h->tune.bdd_fp_staged = sh[2];
            const float a = timed(fwd);
            if (a < 0.f) {
                st = -1;
                break;
            }
            if (a < best_ms) {
                best_ms = a;
                best.bdd_fp_cols = sh[0];
                best.bdd_fp_rows = sh[1];
                best.bdd_fp_staged = sh[2];
            }
        }
    }
    if (e == cudaSuccess && st == OMB_OK && h->desc.bp_type == 5) {
        float best_ms = 3.4e38f;
        // (voxels along z, warps per block, staged); the staged kernel has 8 or 16 voxels and 4 warps
        const int shapes[8][3] = {{4, 4, 0}, {4, 8, 0}, {8, 4, 0}, {8, 8, 0}, {16, 4, 0}, {16, 8, 0}, {8, 4, 1},
                                  {16, 4, 1}};
        for (const auto &sh : shapes) {
            h->tune = best;
            h->tune.bdd_bp_z = sh[0];
            h->tune.bdd_bp_rows = sh[1];
            h->tune.bdd_bp_staged = sh[2];
            const float b = timed(bwd);
            if (b < 0.f) {
                st = -1;
                break;
            }
            if (b < best_ms) {
                best_ms = b;
                best.bdd_bp_z = sh[0];
                best.bdd_bp_rows = sh[1];
                best.bdd_bp_staged = sh[2];
            }
        }
    }
    h->tune = (e == cudaSuccess && st == OMB_OK) ? best : saved;
    const std::string keep = g_last_error;
    if (img) cudaFreeAsync(img, s);
    if (back) cudaFreeAsync(back, s);
    if (y) cudaFreeAsync(y, s);
    const cudaError_t es = cudaStreamSynchronize(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "autotune set-up");
    if (st != OMB_OK) {
        g_last_error = keep.empty() ? "autotune: a timed call failed" : keep;
        return st;
    }
    if (es != cudaSuccess) return cuda_fail(es, "autotune");
    if (out) tuning_to(h->tune, out);
    return OMB_OK;
}

int omb_pdhg_iteration(omb_handle *h, float *x, float *x_next, float *u, float *p, const float *y, float tau,
                       float sigma, float theta, float beta, float tv_smooth, int32_t positivity, float *work_meas,
                       float *work_img, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!x || !x_next || !u || !p || !y || !work_meas || !work_img)
        return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_pdhg_iteration");
    if (x == x_next) return set_error(OMB_ERR_INVALID, "x and x_next must be different buffers");
    cudaStream_t s = (cudaStream_t)stream;
    int st = omb_forward(h, -1, x, work_meas, stream);
    if (st != OMB_OK) return st;
    const int64_t m = omb_measurement_count(h, -1);
    st = pdhg_dual(p, work_meas, y, m, sigma, s);
    if (st != OMB_OK) return st;
    st = omb_backward(h, -1, p, work_img, nullptr, OMB_BP_FLOAT_ATOMIC, stream);
    if (st != OMB_OK) return st;
    return pdhg_primal_tv(h->grid, x, work_img, u, x_next, beta, tv_smooth, tau, theta, h->desc.epps, positivity, s);
}

int omb_pdhg_dual(float *p, const float *fp, const float *y, int64_t n, float sigma, void *stream) {
    if (!p || !fp || !y) return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_pdhg_dual");
    if (n < 0) return set_error(OMB_ERR_INVALID, "n must be >= 0");
    return pdhg_dual(p, fp, y, n, sigma, (cudaStream_t)stream);
}

int omb_pdhg_primal(omb_handle *h, const float *x, const float *rhs, float *u, float *x_next, float tau, float theta,
                    float beta, float tv_smooth, int32_t positivity, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!x || !rhs || !u || !x_next) return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_pdhg_primal");
    if (x == x_next) return set_error(OMB_ERR_INVALID, "x and x_next must be different buffers");
    return pdhg_primal_tv(h->grid, x, rhs, u, x_next, beta, tv_smooth, tau, theta, h->desc.epps, positivity,
                          (cudaStream_t)stream);
}

size_t omb_power_workspace_bytes(void) { return 2 * dot_workspace_bytes(); }

int omb_power_method(omb_handle *h, int32_t n_iter, float *x, float *work_meas, float *work_img, void *work,
                     double *out_host, void *stream) {
    if (!h) return set_error(OMB_ERR_INVALID, "handle is NULL");
    if (!x || !work_meas || !work_img || !work || !out_host)
        return set_error(OMB_ERR_INVALID, "NULL buffer passed to omb_power_method");
    if (n_iter < 1) return set_error(OMB_ERR_INVALID, "n_iter must be >= 1");
    cudaStream_t s = (cudaStream_t)stream;
    double *wl = static_cast<double *>(work);
    double *wn = wl + dot_workspace_bytes() / sizeof(double);
    const int64_t n = h->n_img;
    int st = OMB_OK;
    for (int it = 0; it < n_iter && st == OMB_OK; ++it) {
        st = omb_forward(h, -1, x, work_meas, stream);
        if (st == OMB_OK) st = omb_backward(h, -1, work_meas, work_img, nullptr, OMB_BP_FLOAT_ATOMIC, stream);
        if (st == OMB_OK && it == n_iter - 1) st = dot2(work_img, x, n, wl, s);  // (A^T A x).x and x.x
        if (st == OMB_OK) st = dot2(work_img, work_img, n, wn, s);
        if (st == OMB_OK) st = normalize_into(x, work_img, n, wn + dot_workspace_bytes() / sizeof(double) - 2, s);
    }
    if (st != OMB_OK) return st;
    double d[2];
    OMB_CUDA_TRY(cudaMemcpyAsync(d, wl + dot_workspace_bytes() / sizeof(double) - 2, sizeof(d), cudaMemcpyDeviceToHost, s));
    OMB_CUDA_TRY(cudaStreamSynchronize(s));
    *out_host = d[0] / d[1];
    return OMB_OK;
}

int omb_loglik(const float *y, const float *fp, int64_t n, float epps, double *out_host, void *work, void *stream) {
    if (!y || !fp) return set_error(OMB_ERR_INVALID, "y/fp pointer is NULL");
    if (n < 0) return set_error(OMB_ERR_INVALID, "n must be >= 0");
    return loglik(y, fp, n, epps, out_host, work, (cudaStream_t)stream);
}

size_t omb_reduce_workspace_bytes(int64_t n) { return reduce_workspace_bytes(n); }


// ---------------------------------------------------------------------------
// Batches of independent CT geometries (one persistent launch per direction)
// ---------------------------------------------------------------------------

struct omb_batch {
    int device = 0;
    int n = 0;
    std::vector<int64_t> img_off, meas_off;  // n + 1 cumulative offsets
    float *d_geom = nullptr;                 // all items' xy and z arrays
    BatchItem *d_items = nullptr;
    int2 *d_work = nullptr;
    int n_work = 0;
    int *d_counter = nullptr;
};

int omb_batch_destroy(omb_batch *b) {
    if (!b) return OMB_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != b->device) cudaSetDevice(b->device);
    cudaFree(b->d_geom);
    cudaFree(b->d_items);
    cudaFree(b->d_work);
    cudaFree(b->d_counter);
    if (prev != b->device) cudaSetDevice(prev);
    delete b;
    return OMB_OK;
}

int omb_batch_create(const omb_geometry_desc *descs, int32_t n, omb_batch **out) {
    if (!out) return set_error(OMB_ERR_INVALID, "output batch pointer is NULL");
    *out = nullptr;
    if (!descs || n < 1) return set_error(OMB_ERR_INVALID, "a batch needs at least one geometry");
    for (int i = 0; i < n; ++i) {
        const int st = validate(descs + i);
        if (st != OMB_OK) return set_error(st, "batch item " + std::to_string(i) + ": " + g_last_error);
        const omb_geometry_desc &d = descs[i];
        if (d.modality != OMB_CT_PANEL || d.fp_type != 1 || d.bp_type != 1 || d.tof_bins != 1)
            return set_error(OMB_ERR_UNSUPPORTED, "batch item " + std::to_string(i) +
                                                      ": batches take CT geometries with projector type 1, no TOF");
        if (d.n_proj * (int64_t)d.n_rows_d * d.n_cols_d >= (1ll << 31))
            return set_error(OMB_ERR_UNSUPPORTED, "batch item " + std::to_string(i) + ": too many rays");
    }
    omb_batch *b = new omb_batch();
    cudaGetDevice(&b->device);
    b->n = n;
    b->img_off.assign(n + 1, 0);
    b->meas_off.assign(n + 1, 0);
    int64_t geom_floats = 0;
    for (int i = 0; i < n; ++i) {
        const omb_geometry_desc &d = descs[i];
        b->img_off[i + 1] = b->img_off[i] + (int64_t)d.nx * d.ny * d.nz;
        b->meas_off[i + 1] = b->meas_off[i] + d.n_proj * (int64_t)d.n_rows_d * d.n_cols_d;
        geom_floats += d.n_xy + d.n_z;
    }
    auto fail = [&](cudaError_t e, const char *what) {
        omb_batch_destroy(b);
        return cuda_fail(e, what);
    };
    cudaError_t e = cudaMalloc(&b->d_geom, geom_floats * sizeof(float));
    if (e != cudaSuccess) return fail(e, "cudaMalloc batch geometry");
    std::vector<BatchItem> items((size_t)n);
    int64_t pos = 0;
    for (int i = 0; i < n; ++i) {
        const omb_geometry_desc &d = descs[i];
        float *xy = b->d_geom + pos, *z = xy + d.n_xy;
        if ((e = cudaMemcpy(xy, d.xy, d.n_xy * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(e, "upload batch xy");
        if ((e = cudaMemcpy(z, d.z, d.n_z * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(e, "upload batch z");
        pos += d.n_xy + d.n_z;
        BatchItem &it = items[(size_t)i];
        Grid &g = it.g;
        g.nx = (int)d.nx; g.ny = (int)d.ny; g.nz = (int)d.nz;
        g.dx = d.dx; g.dy = d.dy; g.dz = d.dz;
        g.bx = d.bx; g.by = d.by; g.bz = d.bz;
        g.mx = d.bx + (float)d.nx * d.dx;
        g.my = d.by + (float)d.ny * d.dy;
        g.mz = d.bz + (float)d.nz * d.dz;
        RaySet &rs = it.rs;
        rs = RaySet{};
        rs.xy = xy;
        rs.z = z;
        rs.modality = OMB_CT_PANEL;
        rs.n_rows = (int)d.n_rows_d;
        rs.n_cols = (int)d.n_cols_d;
        rs.pitch_x = d.dpitch_x;
        rs.pitch_y = d.dpitch_y;
        rs.proj0 = 0;
        rs.n_proj = d.n_proj;
        rs.m_size = b->meas_off[i + 1] - b->meas_off[i];
        rs.stype = 0;
        rs.n_subsets = 1;
        rs.cur_subset = 0;
        it.img_off = b->img_off[i];
        it.meas_off = b->meas_off[i];
    }
    // chunks of one block's rays, the costliest items (rays x walk length) first
    std::vector<int> order((size_t)n);
    for (int i = 0; i < n; ++i) order[(size_t)i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int c) {
        const double ca = (double)items[(size_t)a].rs.m_size * (descs[a].nx + descs[a].ny);
        const double cc = (double)items[(size_t)c].rs.m_size * (descs[c].nx + descs[c].ny);
        return ca > cc;
    });
    std::vector<int2> work;
    for (int i : order)
        for (int64_t r = 0; r < items[(size_t)i].rs.m_size; r += 32) work.push_back(make_int2(i, (int)r));  // warp chunks
    b->n_work = (int)work.size();
    if ((e = cudaMalloc(&b->d_items, items.size() * sizeof(BatchItem))) != cudaSuccess) return fail(e, "cudaMalloc batch items");
    if ((e = cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "upload batch items");
    if ((e = cudaMalloc(&b->d_work, work.size() * sizeof(int2))) != cudaSuccess) return fail(e, "cudaMalloc batch work");
    if ((e = cudaMemcpy(b->d_work, work.data(), work.size() * sizeof(int2), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "upload batch work");
    if ((e = cudaMalloc(&b->d_counter, sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc batch counter");
    *out = b;
    return OMB_OK;
}

int64_t omb_batch_image_offset(const omb_batch *b, int32_t item) {
    if (!b || item < 0 || item > b->n) return -1;
    return b->img_off[(size_t)item];
}

int64_t omb_batch_measurement_offset(const omb_batch *b, int32_t item) {
    if (!b || item < 0 || item > b->n) return -1;
    return b->meas_off[(size_t)item];
}

int omb_batch_forward(omb_batch *b, const float *images, float *y, void *stream) {
    if (!b) return set_error(OMB_ERR_INVALID, "batch is NULL");
    if (!images || !y) return set_error(OMB_ERR_INVALID, "images/y pointer is NULL");
    return batch_project(b->d_items, b->d_work, b->n_work, b->d_counter, images, y, false, (cudaStream_t)stream);
}

int omb_batch_backward(omb_batch *b, const float *y, float *images, void *stream) {
    if (!b) return set_error(OMB_ERR_INVALID, "batch is NULL");
    if (!images || !y) return set_error(OMB_ERR_INVALID, "images/y pointer is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    OMB_CUDA_TRY(cudaMemsetAsync(images, 0, b->img_off[(size_t)b->n] * sizeof(float), s));
    return batch_project(b->d_items, b->d_work, b->n_work, b->d_counter, y, images, true, s);
}

}  // extern "C"

extern "C" int omb_precond_image(omb_handle *h, float *d, float *work_img, void *stream) {
    if (!h || !d || !work_img) return set_error(OMB_ERR_INVALID, "NULL pointer passed to omb_precond_image");
    cudaStream_t s = (cudaStream_t)stream;
    const int S = h->desc.n_subsets;
    for (int s_ = 0; s_ < S; ++s_) {
        int st = sensitivity_raw(h, s_, s_ == 0 ? d : work_img, s);
        if (st == OMB_OK && s_ > 0) st = add_into(d, work_img, h->n_img, s);
        if (st != OMB_OK) return st;
    }
    return precond_finish(d, h->n_img, S, s);
}
