// Shared host/device definitions of the omega_b200 projector library.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/omega_b200.h"

namespace omb {

// Records `msg` as the calling thread's last error and returns `code`.
int set_error(int code, const std::string &msg);
// Turns a CUDA error into OMB_ERR_CUDA with a message naming `what`.
int cuda_fail(cudaError_t e, const char *what);

#define OMB_CUDA_TRY(call)                                   \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return ::omb::cuda_fail(_e, #call); \
    } while (0)

#define OMB_LAUNCH_CHECK(what)                                  \
    do {                                                        \
        cudaError_t _e = cudaGetLastError();                    \
        if (_e != cudaSuccess) return ::omb::cuda_fail(_e, what); \
    } while (0)

// Voxel grid of one image volume.
struct Grid {
    int nx, ny, nz;
    float dx, dy, dz;
    float bx, by, bz;     // lower FOV corner
    float mx, my, mz;     // upper FOV corner b + N*d
};

// Where one launch's rays come from.  A launch covers `n_proj` consecutive
// sinograms/projections starting at global position `proj0` (subset order),
// or, for measurement-level PET subsets (types 1, 2, 4, 5), `m_size`
// measurements of subset `cur_subset` spread over the whole sinogram.
struct RaySet {
    const float *xy;
    const float *z;
    int modality;       // omb_modality
    int n_rows;         // Ndist / detector rows
    int n_cols;         // Nang / detector columns
    int64_t proj0;
    int64_t n_proj;
    int64_t m_size;     // rays in this launch (TOF bin stride)
    int stype;          // 0: whole sinograms; 1, 2, 4, 5: measurement-level
    int n_subsets;
    int cur_subset;
    float pitch_x, pitch_y;
    const uint16_t *tr; // OMB_PET_INDEXED: transaxial index pairs of all events
    const uint16_t *ax; // OMB_PET_INDEXED: axial index pairs of all events
    int nr_xy, nr_z;    // PET multi-ray: rays per LOR transaxially / axially (1, 1 = one ray)
    float cr_xy, cr_z;  // crystal sizes the rays are spread over (mm)
    const float *w;     // PET: multiplicative weight of each of the launch's rays, or NULL
    const float *mu;    // PET: attenuation image (1/mm), or NULL
};

// Projector types 2 / 3: the tube of response.
struct Orth {
    int type;            // 2 orthogonal distance, 3 volume of intersection
    float width;         // type 2: tube width (FWHM-like, mm); type 3: tube radius (mm)
    int xy, z;           // tube spread transaxially / axially
    float bmin, bmax, vmax;
    const float *v;      // type 3: intersection volume per 1/1000 mm of distance above bmin
    int nv;
};

// One reconstruction of a batch projected by one persistent launch: its
// grid, its rays and where its image and measurements start in the batch's
// concatenated buffers.
struct BatchItem {
    Grid g;
    RaySet rs;
    int64_t img_off;
    int64_t meas_off;
};

// A batch of frames (images and their measurement vectors) processed by one
// launch; frame f's image starts at img + f*img_stride and its measurements
// at meas + f*meas_stride.
struct Frames {
    int n;
    const float *img_in;   // forward: input images
    const __nv_bfloat16 *img_in16;  // forward: BF16 copies of the images (read instead of img_in when set)
    float *img;            // backward: output images
    int64_t img_stride;
    const float *meas;     // backward: input measurements
    float *meas_out;       // forward: output measurements
    int64_t meas_stride;
    float *ilv;            // scratch of ceil(n / FB) * FB images in voxel-interleaved order, or NULL
    int64_t ilv_floats;    // its capacity
};

struct Tof {
    int nbins;
    float sigma_inv;
    float sigma_coef;   // 1/sqrt(2 pi) / sigma
    float epps;
    const float *centers;
};

// Per-projection constants of the distance-driven backprojection: a
// projective map from world coordinates q to continuous detector pixel-edge
// coordinates, u = (au.q + au0) / (c.q + 1), v = (av.q + av0) / (c.q + 1),
// plus the source position and which axis the footprint mid-plane follows.
struct BddProj {
    float au[3], au0;
    float av[3], av0;
    float c[3];
    float s[3];
    int ysl;    // |s.x| <= |s.y|: voxel mid-plane spans x and z
    int spos;   // sign of the source's dominant coordinate (s.y if ysl, else s.x) > 0
    float k;    // the ray s -> q meets the panel at s + (k / (c.q + 1)) (q - s)
    float pad[3];
};

// The same map in FP64 (the values BddProj rounds), for re-basing it to one
// thread block: evaluated in FP32 at pixel coordinates of several hundred the
// map carries ~3e-5 pixels of rounding, which moves a backprojection by
// ~1e-5 relative L2 at 512^2 panels; re-based it carries ~2e-6.
struct BddMap64 {
    double au[3], au0;
    double av[3], av0;
    double c[3], pad;
};

// A projection's map re-based to one block of voxels: with d = q - p0 (p0 a
// corner of the block) and integer pixel origins (U0, V0),
//   u - U0 = (au . d + nu0) / (c . d + d0),  v - V0 = (av . d + nv0) / (c . d + d0),
// coefficients rounded to FP32 from FP64.  Also carries what the voxel loop
// needs of BddProj (source, slice orientation) so it reads no global memory.
// Laid out as 16-byte vectors so a thread reads it with five vector loads:
//   u = (au.x, au.y, au.z, nu0), v = (av.x, av.y, av.z, nv0),
//   c = (c.x, c.y, c.z, d0), s = (source x, y, z, float(U0)),
//   o = (U0, V0, ysl, spos).
struct alignas(16) BddMapR {
    float4 u, v, c, s;
    int4 o;
};

// Re-bases M to the block corner p0 with pixel origins (U0, V0), in FP64.
__device__ __forceinline__ void bdd_rebase(BddMapR &R, const BddMap64 &M, const BddProj &P, double p0x, double p0y,
                                           double p0z, int U0, int V0) {
    const double D0 = fma(M.c[0], p0x, fma(M.c[1], p0y, fma(M.c[2], p0z, 1.0)));
    const double Nu = fma(M.au[0], p0x, fma(M.au[1], p0y, fma(M.au[2], p0z, M.au0)));
    const double Nv = fma(M.av[0], p0x, fma(M.av[1], p0y, fma(M.av[2], p0z, M.av0)));
    const double u0 = (double)U0, v0 = (double)V0;
    R.u = make_float4((float)(M.au[0] - u0 * M.c[0]), (float)(M.au[1] - u0 * M.c[1]), (float)(M.au[2] - u0 * M.c[2]),
                      (float)(Nu - u0 * D0));
    R.v = make_float4((float)(M.av[0] - v0 * M.c[0]), (float)(M.av[1] - v0 * M.c[1]), (float)(M.av[2] - v0 * M.c[2]),
                      (float)(Nv - v0 * D0));
    R.c = make_float4((float)M.c[0], (float)M.c[1], (float)M.c[2], (float)D0);
    R.s = make_float4(P.s[0], P.s[1], P.s[2], (float)U0);
    R.o = make_int4(U0, V0, P.ysl, P.spos);
}

// Pixel origin of a block's re-based map: the lowest row / column the
// float map sends any of the block's 8 corners to, minus one, clamped into
// the panel, the row rounded down to a multiple of 4 (the staged kernel's
// detector box starts there; the box load needs a 16-byte aligned start).
__device__ __forceinline__ int2 bdd_block_origin(float umin, float vmin, int nr, int nc) {
    int r = (int)floorf(fmaxf(umin - 1.f, 0.f));
    r = min(r, nr - 1) & ~3;
    int c = (int)floorf(fmaxf(vmin - 1.f, 0.f));
    c = min(c, nc - 1);
    return make_int2(r, c);
}

// The float map at one corner of a block (the staged kernel's box corners).
__device__ __forceinline__ float2 bdd_corner_uv(const BddProj &P, float cx, float cy, float cz) {
    const float den = 1.f / fmaf(P.c[0], cx, fmaf(P.c[1], cy, fmaf(P.c[2], cz, 1.f)));
    return make_float2(fmaf(P.au[0], cx, fmaf(P.au[1], cy, fmaf(P.au[2], cz, P.au0))) * den,
                       fmaf(P.av[0], cx, fmaf(P.av[1], cy, fmaf(P.av[2], cz, P.av0))) * den);
}

// Pixel coordinates (u, v) of world point p under M, FP64.
__device__ __forceinline__ void bdd_map_at(const BddMap64 &M, double px, double py, double pz, double &u, double &v) {
    const double D = fma(M.c[0], px, fma(M.c[1], py, fma(M.c[2], pz, 1.0)));
    u = fma(M.au[0], px, fma(M.au[1], py, fma(M.au[2], pz, M.au0))) / D;
    v = fma(M.av[0], px, fma(M.av[1], py, fma(M.av[2], pz, M.av0))) / D;
}

// Launch shapes the autotuner chooses between (per handle).
struct Tuning {
    int siddon_blocks_per_sm = 8;   // grid-stride grid of the Siddon kernels: blocks per SM
    int siddon_frames = 8;          // most frames sharing one ray walk (1, 2, 4, 8)
    int bdd_fp_cols = 8;            // type-5 forward: detector columns per thread (8, 16)
    int bdd_bp_z = 8;               // type-5 backward: voxels along z per thread (4, 8, 16)
    int bdd_fp_rows = 8;            // type-5 forward: warps per block (4, 8)
    int bdd_bp_rows = 8;            // type-5 backward: warps per block (4, 8)
    int siddon_layout = 1;          // frame batches: 0 = frame-major reads/atomics, 1 = voxel-interleaved
    int siddon_fp_steps = 4;        // non-TOF forward walks: crossings gathered per batched step (1, 2, 4)
    int bdd_fp_staged = 1;          // type-5 forward: image boxes staged by TMA (with 8 columns per thread)
    int bdd_bp_staged = 1;          // type-5 backward: detector boxes staged by TMA (with 8 or 16 voxels per thread)
    int siddon_bp_matrix = 0;       // type-1 non-TOF backprojection through a resident transposed system matrix
};

// Read-only image load as float from an FP32 or BF16 array.
__device__ __forceinline__ float ld_img(const float *p) { return __ldg(p); }
__device__ __forceinline__ float ld_img(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }

constexpr int kMaxTofBins = 16;
// Fixed-point scale of the int64 backprojection mode (the reference's TH).
constexpr double kFixedScale = 1e11;
constexpr int kBlock = 256;

inline int num_sms() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

// Grid size for a grid-stride kernel over `n` items: at most `per_sm`
// resident blocks on every SM.
inline unsigned grid_for(int64_t n, int per_sm = 8, int block = kBlock) {
    int64_t need = (n + block - 1) / block;
    int64_t cap = (int64_t)num_sms() * per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

}  // namespace omb
