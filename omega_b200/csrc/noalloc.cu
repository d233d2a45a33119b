// Allocation-free variant of the int64 fixed-point backprojection.
//
// Some callers cannot allocate device memory: their device memory belongs to
// another allocator (a framework's caching pool or a scanner pipeline that
// reserves its budget at start-up), so an extra cudaMalloc either fails or
// breaks the budget they were given.  omb_backward_fixed64_noalloc serves
// them: the caller passes every input and output (geometry arrays included)
// as device buffers, and the int64 accumulators live in a fixed-size
// file-scope device array instead of a per-handle allocation.
//
// The array is OMB_NOALLOC_MAX_VOXELS image voxels + as many sensitivity
// voxels, 8 bytes each (16 MiB); every GPU that loads this library holds it
// until the process exits.  All calls share it and it keeps the previous
// call's contents, so each call clears the part it uses first, and calls
// whose work overlaps on the GPU (different streams, or different host
// threads on the same device) race on it.
#include <mutex>

#include "kernels.h"

namespace omb {

static __device__ __align__(256) unsigned long long g_noalloc_acc[2 * (size_t)OMB_NOALLOC_MAX_VOXELS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned long long *g_acc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_acc on the current device.  The symbol's name
// in host code is a host-side stand-in, not a device address, so the address
// is looked up once per device (with that device current) and cached.
int scratch_for_current_device(unsigned long long **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error(OMB_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_acc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_acc);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_acc)");
        g_acc_ptr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_acc_ptr[dev];
    return OMB_OK;
}

int check_desc(const omb_geometry_desc *d, int32_t subset) {
    if (!d) return set_error(OMB_ERR_INVALID, "geometry descriptor is NULL");
    if (d->struct_size != sizeof(omb_geometry_desc) || d->abi_version != OMB_ABI_VERSION)
        return set_error(OMB_ERR_INVALID, "omb_geometry_desc struct_size/abi_version do not match this library");
    if (d->modality != OMB_PET_SINOGRAM && d->modality != OMB_CT_PANEL)
        return set_error(OMB_ERR_INVALID, "modality must be OMB_PET_SINOGRAM or OMB_CT_PANEL");
    if (d->bp_type != 1) return set_error(OMB_ERR_UNSUPPORTED, "the allocation-free backprojection is projector type 1");
    if (d->n_rays_xy > 1 || d->n_rays_z > 1)
        return set_error(OMB_ERR_UNSUPPORTED, "the allocation-free backprojection takes one ray per LOR");
    if (d->nx == 0 || d->ny == 0 || d->nz == 0) return set_error(OMB_ERR_INVALID, "image size must be positive");
    const uint64_t n_vox = (uint64_t)d->nx * d->ny * d->nz;
    if (n_vox > (uint64_t)OMB_NOALLOC_MAX_VOXELS)
        return set_error(OMB_ERR_UNSUPPORTED, "image of " + std::to_string(n_vox) +
                                                  " voxels exceeds the allocation-free limit of " +
                                                  std::to_string((uint64_t)OMB_NOALLOC_MAX_VOXELS) + " voxels");
    if (!(d->dx > 0.f) || !(d->dy > 0.f) || !(d->dz > 0.f)) return set_error(OMB_ERR_INVALID, "voxel size must be positive");
    if (d->n_rows_d == 0 || d->n_cols_d == 0 || d->n_proj <= 0) return set_error(OMB_ERR_INVALID, "detector/projection counts must be positive");
    if (d->n_subsets < 1 || !d->n_meas) return set_error(OMB_ERR_INVALID, "n_subsets/n_meas invalid");
    if (subset < -1 || subset >= d->n_subsets) return set_error(OMB_ERR_INVALID, "subset out of range");
    if (!d->xy || !d->z) return set_error(OMB_ERR_INVALID, "xy/z device arrays are NULL");
    if (d->n_subsets > 1 && d->subset_type < 8) {
        if (d->modality != OMB_PET_SINOGRAM)
            return set_error(OMB_ERR_UNSUPPORTED, "measurement-level subset types are PET-only");
        if (d->subset_type != 1 && d->subset_type != 2 && d->subset_type != 4 && d->subset_type != 5)
            return set_error(OMB_ERR_UNSUPPORTED, "subset type not built");
        if (subset < 0) return set_error(OMB_ERR_UNSUPPORTED, "subset -1 needs a whole-sinogram subset type");
    }
    const int64_t nbin = (int64_t)d->n_rows_d * d->n_cols_d;
    if (d->modality == OMB_PET_SINOGRAM) {
        if (d->n_xy != nbin * 4 || d->n_z != d->n_proj * 2) return set_error(OMB_ERR_INVALID, "PET xy/z sizes invalid");
    } else {
        if (d->n_xy != d->n_proj * 6 || d->n_z != d->n_proj * 2) return set_error(OMB_ERR_INVALID, "CT xy/z sizes invalid");
    }
    if (d->tof_bins < 1 || d->tof_bins > kMaxTofBins) return set_error(OMB_ERR_UNSUPPORTED, "tof_bins must be 1-16");
    if (d->tof_bins > 1 && (!d->tof_centers || !(d->sigma_x > 0.f)))
        return set_error(OMB_ERR_INVALID, "TOF needs tof_centers (device) and a positive sigma");
    const int64_t *nm = d->n_meas;
    if (nm[0] != 0) return set_error(OMB_ERR_INVALID, "n_meas[0] must be 0");
    for (int s = 0; s < d->n_subsets; ++s)
        if (nm[s + 1] < nm[s]) return set_error(OMB_ERR_INVALID, "n_meas must be non-decreasing");
    if (!(d->n_subsets > 1 && d->subset_type < 8) && nm[d->n_subsets] != d->n_proj)
        return set_error(OMB_ERR_INVALID, "n_meas[n_subsets] must equal n_proj");
    return OMB_OK;
}

}  // namespace
}  // namespace omb

using namespace omb;

extern "C" int omb_backward_fixed64_noalloc(const omb_geometry_desc *desc, int32_t subset, const float *y,
                                            float *image, float *sens, void *stream) {
    int st = check_desc(desc, subset);
    if (st != OMB_OK) return st;
    if (!y || !image) return set_error(OMB_ERR_INVALID, "y/image pointer is NULL");
    unsigned long long *acc = nullptr;
    st = scratch_for_current_device(&acc);
    if (st != OMB_OK) return st;
    const omb_geometry_desc &d = *desc;
    Grid g{};
    g.nx = (int)d.nx; g.ny = (int)d.ny; g.nz = (int)d.nz;
    g.dx = d.dx; g.dy = d.dy; g.dz = d.dz;
    g.bx = d.bx; g.by = d.by; g.bz = d.bz;
    g.mx = d.bx + (float)d.nx * d.dx;
    g.my = d.by + (float)d.ny * d.dy;
    g.mz = d.bz + (float)d.nz * d.dz;
    Tof tof{};
    tof.nbins = d.tof_bins;
    tof.epps = d.epps;
    tof.sigma_inv = d.tof_bins > 1 ? 1.f / d.sigma_x : 0.f;
    tof.sigma_coef = 0.3989423f * tof.sigma_inv;
    tof.centers = d.tof_centers;
    RaySet rs{};
    rs.xy = d.xy;
    rs.z = d.z;
    rs.modality = d.modality;
    rs.n_rows = (int)d.n_rows_d;
    rs.n_cols = (int)d.n_cols_d;
    rs.pitch_x = d.dpitch_x;
    rs.pitch_y = d.dpitch_y;
    rs.n_subsets = d.n_subsets;
    if (d.n_subsets > 1 && d.subset_type < 8) {
        rs.stype = d.subset_type;
        rs.cur_subset = subset;
        rs.proj0 = 0;
        rs.n_proj = d.n_proj;
        rs.m_size = d.n_meas[subset + 1] - d.n_meas[subset];
    } else {
        rs.stype = 0;
        rs.cur_subset = subset < 0 ? 0 : subset;
        rs.proj0 = subset < 0 ? 0 : d.n_meas[subset];
        rs.n_proj = subset < 0 ? d.n_proj : d.n_meas[subset + 1] - d.n_meas[subset];
        rs.m_size = rs.n_proj * (int64_t)d.n_rows_d * d.n_cols_d;
    }
    const int64_t n = (int64_t)d.nx * d.ny * d.nz;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long *acc_s = sens ? acc + n : nullptr;
    // the array keeps the previous call's sums: clear the part this call uses
    OMB_CUDA_TRY(cudaMemsetAsync(acc, 0, (sens ? 2 : 1) * n * sizeof(unsigned long long), s));
    st = siddon_backward_fixed(g, rs, tof, d.global_factor, y, acc, acc_s, s);
    if (st != OMB_OK) return st;
    st = fixed_to_float(acc, image, n, s);
    if (st == OMB_OK && sens) st = fixed_to_float(acc_s, sens, n, s);
    return st;
}
