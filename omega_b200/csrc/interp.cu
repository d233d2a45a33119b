// Projector type 4: interpolation-based projections.
//
// Forward (PET and CT): the ray from s to d is sampled every dL millimetres
// from its FOV entry point and the image is trilinearly interpolated at each
// sample (projectorType4Forward, projectorType4.cl:84-683, non-Joseph path:
// t-range 392-401, tStep = dL/L, nSteps = floor((tEnd - tStart)/tStep) + 1,
// 467-476).  PET outputs are scaled by global_factor / L (TOTLENGTH), CT
// outputs are the plain sums dL * f(p) (forwardProjectAF, general_opencl_
// functions.h:1961-1967).  TOF bins use the trapezoid weights of the type-1
// projector with element length dL (TOFLoop 1103-1117).
//
// Backward, PET: the same march, each sample's weight dL * gf / L * y added to
// the voxel that contains it (index truncated per axis; the flat index 0 is
// skipped, as the reference's `local_ind <= 0` test does) with float or
// int64 fixed-point atomics (projectorType4.cl:579-599, rhs 1212-1275).
//
// Backward, CT: voxel-driven; each voxel centre is projected onto every
// panel, the projection is bilinearly interpolated there (clamped to the
// edge, zero outside the panel) and weighted by L^3 / |v|^2 * kerroin with L
// the source-to-panel distance along the ray and v the source-to-voxel vector
// (projectorType4Backward, projectorType4.cl:718-1100; the sensitivity sums
// the weights where the interpolated value is nonzero).
//
// Differences from the reference kernels, all deliberate:
//  * the reference samples the image and the projections through linear
//    filtering textures, whose weights carry 8 fractional bits; here the
//    trilinear / bilinear weights are exact FP32;
//  * the ray set-up (t-range, step, sample count) runs in FP64 with every
//    operation rounded separately, so the sample count is reproducible
//    (rays whose FOV chord is an exact multiple of dL otherwise gain or lose
//    their last sample to rounding); samples are placed at t0 + n * tStep
//    (one FMA from the step index) instead of a running sum re-anchored every
//    64 steps;
//  * the CT backprojection evaluates the panel coordinates through the same
//    FP64-built projective map as the type-5 backprojection instead of the
//    FP32 plane intersection (identical in exact arithmetic).
#include "kernels.h"
#include "siddon.cuh"

namespace omb {

// One ray's samples: texel coordinates (voxel centres at integers) of sample
// n are c + n * step per axis.
struct March {
    float cx, cy, cz;
    float sx, sy, sz;
    unsigned n;
    float L;
    float D0;  // TOF: distance of the first sample from the LOR centre (signed)
    double ts, tstep;  // first sample and step along the ray (t in [0, 1] from s to d)
};

// b + N*d rounded to float32 from a double sum, as the reference's host code
// forms bmax (projfunctions.py:397-399).
__device__ __forceinline__ double upper_edge(float b, int n, float d) {
    return (double)(float)__dadd_rn((double)b, __dmul_rn((double)n, (double)d));
}

__device__ __forceinline__ bool march_setup(const Grid &g, const Ray &ray, float dL, March &m) {
    const double sx = ray.s.x, sy = ray.s.y, sz = ray.s.z;
    const double vx = __dsub_rn((double)ray.d.x, sx), vy = __dsub_rn((double)ray.d.y, sy),
                 vz = __dsub_rn((double)ray.d.z, sz);
    const double bx = g.bx, by = g.by, bz = g.bz;
    const double t0x = __ddiv_rn(__dsub_rn(bx, sx), vx), t1x = __ddiv_rn(__dsub_rn(upper_edge(g.bx, g.nx, g.dx), sx), vx);
    const double t0y = __ddiv_rn(__dsub_rn(by, sy), vy), t1y = __ddiv_rn(__dsub_rn(upper_edge(g.by, g.ny, g.dy), sy), vy);
    const double t0z = __ddiv_rn(__dsub_rn(bz, sz), vz), t1z = __ddiv_rn(__dsub_rn(upper_edge(g.bz, g.nz, g.dz), sz), vz);
    const double ts = fmax(fmax(fmin(t0x, t1x), fmin(t0y, t1y)), fmin(t0z, t1z));
    const double te = fmin(fmin(fmax(t0x, t1x), fmax(t0y, t1y)), fmax(t0z, t1z));
    if (!(ts < te)) return false;
    const double L = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz)));
    const double tstep = __ddiv_rn((double)dL, L);
    const double q = __ddiv_rn(__dsub_rn(te, ts), tstep);
    if (!(q >= 0.0) || q >= 4.0e9) return false;
    m.n = (unsigned)q + 1u;
    m.L = (float)L;
    m.ts = ts;
    m.tstep = tstep;
    const double ix = 1.0 / (double)g.dx, iy = 1.0 / (double)g.dy, iz = 1.0 / (double)g.dz;
    m.cx = (float)((sx + vx * ts - bx) * ix - 0.5);
    m.cy = (float)((sy + vy * ts - by) * iy - 0.5);
    m.cz = (float)((sz + vz * ts - bz) * iz - 0.5);
    m.sx = (float)(vx * tstep * ix);
    m.sy = (float)(vy * tstep * iy);
    m.sz = (float)(vz * tstep * iz);
    m.D0 = (float)(fabs(ts) * L - 0.5 * L);
    return true;
}

// Voxel index of a position in voxel units: truncation toward zero, negative
// and NaN to 0 (the reference's CUINT_rtz of p * N).
__device__ __forceinline__ unsigned voxel_of(double p) {
    return p > 0.0 ? (p < 4294967295.0 ? (unsigned)p : 4294967295u) : 0u;
}

// Trilinear interpolation with clamp-to-edge addressing; (x, y, z) are texel
// coordinates (voxel centres at integers).
template <typename T>
__device__ __forceinline__ float trilinear(const T *__restrict__ img, const Grid &g, float x, float y, float z) {
    x = fminf(fmaxf(x, -1.f), (float)g.nx);
    y = fminf(fmaxf(y, -1.f), (float)g.ny);
    z = fminf(fmaxf(z, -1.f), (float)g.nz);
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const float ax = x - fx, ay = y - fy, az = z - fz;
    const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    const int x0 = min(max(ix, 0), g.nx - 1), x1 = min(max(ix + 1, 0), g.nx - 1);
    const int64_t nxy = (int64_t)g.nx * g.ny;
    const int64_t y0 = (int64_t)min(max(iy, 0), g.ny - 1) * g.nx, y1 = (int64_t)min(max(iy + 1, 0), g.ny - 1) * g.nx;
    const int64_t z0 = (int64_t)min(max(iz, 0), g.nz - 1) * nxy, z1 = (int64_t)min(max(iz + 1, 0), g.nz - 1) * nxy;
    const float v000 = ld_img(img + x0 + y0 + z0), v100 = ld_img(img + x1 + y0 + z0);
    const float v010 = ld_img(img + x0 + y1 + z0), v110 = ld_img(img + x1 + y1 + z0);
    const float v001 = ld_img(img + x0 + y0 + z1), v101 = ld_img(img + x1 + y0 + z1);
    const float v011 = ld_img(img + x0 + y1 + z1), v111 = ld_img(img + x1 + y1 + z1);
    const float c00 = fmaf(ax, v100 - v000, v000), c10 = fmaf(ax, v110 - v010, v010);
    const float c01 = fmaf(ax, v101 - v001, v001), c11 = fmaf(ax, v111 - v011, v011);
    const float c0 = fmaf(ay, c10 - c00, c00), c1 = fmaf(ay, c11 - c01, c01);
    return fmaf(az, c1 - c0, c0);
}

// At most 80 registers (3 CTAs of 256 per SM): with the TOF weights' four
// exponentials in flight per bin the forward projection otherwise takes 86
// and falls to 2 CTAs (67.3 against 72.8 ms for 16 subsets x 15 bins).
template <int NB, typename T>
__global__ void __launch_bounds__(kBlock, 3) k_interp_fp(Grid g, RaySet rs, Tof tof, float gf, float dL, const T *__restrict__ img,
                            float *__restrict__ y) {
    const bool pet = rs.modality != OMB_CT_PANEL;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        float ax[NB];
#pragma unroll
        for (int to = 0; to < NB; ++to) ax[to] = 0.f;
        const Ray ray = load_ray(rs, r);
        March m;
        float temp = 0.f;
        if (march_setup(g, ray, dL, m)) {
            temp = pet ? (1.f / m.L) * gf : 1.f;
            const float ddsign = sgnf(m.D0);
            float w[NB > 1 ? NB : 1];
            for (unsigned ii = 0; ii < m.n; ++ii) {
                const float fi = (float)ii;
                const float val =
                    dL * trilinear(img, g, fmaf(fi, m.sx, m.cx), fmaf(fi, m.sy, m.cy), fmaf(fi, m.sz, m.cz));
                if (NB == 1) {
                    ax[0] += val;
                } else {
                    const float D = fmaf(-fi * dL, ddsign, m.D0);
                    const float tsum = tof_weights<NB>(tof, ddsign, dL, D, w);
                    const float dX = val / tsum;
#pragma unroll
                    for (int to = 0; to < NB; ++to) ax[to] = fmaf(w[to], dX, ax[to]);
                }
            }
        }
#pragma unroll
        for (int to = 0; to < NB; ++to) y[r + to * rs.m_size] = ax[to] * temp;
    }
}

// Ray-driven PET backprojection.  FIXED: int64 fixed-point accumulators
// (order independent, identical run to run); else float atomics.  y == NULL
// backprojects ones; img == NULL (float mode) keeps only the sensitivity.
template <int NB, bool SENS, bool FIXED>
__global__ void k_interp_bp(Grid g, RaySet rs, Tof tof, float gf, float dL,
                                                      const float *__restrict__ y, float *__restrict__ img,
                                                      float *__restrict__ sens, unsigned long long *__restrict__ acc,
                                                      unsigned long long *__restrict__ acc_s) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const unsigned nx = (unsigned)g.nx, nxy = (unsigned)g.nx * (unsigned)g.ny;
    const unsigned ntot = nxy * (unsigned)g.nz;
    const double bx = g.bx, by = g.by, bz = g.bz;
    const double ivx = __ddiv_rn(1.0, (double)g.dx), ivy = __ddiv_rn(1.0, (double)g.dy),
                 ivz = __ddiv_rn(1.0, (double)g.dz);
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.m_size; r += stride) {
        float ax[NB];
        bool any = SENS || y == nullptr;
#pragma unroll
        for (int to = 0; to < NB; ++to) {
            ax[to] = y ? __ldg(y + r + to * rs.m_size) : 1.f;
            any |= ax[to] != 0.f;
        }
        if (!any) continue;
        const Ray ray = load_ray(rs, r);
        March m;
        if (!march_setup(g, ray, dL, m)) continue;
        const float le = dL * ((1.f / m.L) * gf);
        const float ddsign = sgnf(m.D0);
        float w[NB > 1 ? NB : 1];
        // TOF distance: advanced only after samples that land in the image (the
        // reference's loop skips its decrement together with the sample)
        unsigned kd = 0;
        // The voxel of a sample is decided in FP64 with separately rounded
        // operations: samples of axis-parallel rays fall exactly on voxel
        // faces, where an FP32 position picks either neighbour.
        const double sx = ray.s.x, sy = ray.s.y, sz = ray.s.z;
        const double vx = __dsub_rn((double)ray.d.x, sx), vy = __dsub_rn((double)ray.d.y, sy),
                     vz = __dsub_rn((double)ray.d.z, sz);
        for (unsigned ii = 0; ii < m.n; ++ii) {
            const double t = __dadd_rn(m.ts, __dmul_rn((double)ii, m.tstep));
            const unsigned ux = voxel_of(__dmul_rn(__dsub_rn(__dadd_rn(sx, __dmul_rn(vx, t)), bx), ivx));
            const unsigned uy = voxel_of(__dmul_rn(__dsub_rn(__dadd_rn(sy, __dmul_rn(vy, t)), by), ivy));
            const unsigned uz = voxel_of(__dmul_rn(__dsub_rn(__dadd_rn(sz, __dmul_rn(vz, t)), bz), ivz));
            const unsigned ind = ux + uy * nx + uz * nxy;
            float yax, val;
            if (NB == 1) {
                yax = ax[0] * le;
                val = le;
                if (isnan(le)) yax = 0.f;
            } else {
                const float D = fmaf(-(float)kd * dL, ddsign, m.D0);
                const float tsum = tof_weights<NB>(tof, ddsign, dL, D, w);
                const float dX = le / tsum;
                yax = 0.f;
                val = 0.f;
#pragma unroll
                for (int to = 0; to < NB; ++to) {
                    const float a = dX * w[to];
                    val += a;
                    yax += a * ax[to];
                }
            }
            if (ind == 0u || ind >= ntot) continue;
            ++kd;
            if (FIXED) {
                const long long q = (long long)((double)yax * kFixedScale);
                if (q != 0) atomicAdd(acc + ind, (unsigned long long)q);
                if (SENS) {
                    const long long qs = (long long)((double)val * kFixedScale);
                    if (qs != 0) atomicAdd(acc_s + ind, (unsigned long long)qs);
                }
            } else {
                if (img != nullptr && yax != 0.f) atomicAdd(img + ind, yax);
                if (SENS && val != 0.f) atomicAdd(sens + ind, val);
            }
        }
    }
}

// Bilinear interpolation of one projection (rows fastest) with clamp-to-edge
// addressing at texel coordinates (u, v) (pixel centres at integers).
__device__ __forceinline__ float bilinear(const float *__restrict__ yp, int nr, int nc, float u, float v) {
    const float fu = floorf(u), fv = floorf(v);
    const float au = u - fu, av = v - fv;
    const int iu = (int)fu, iv = (int)fv;
    const int u0 = min(max(iu, 0), nr - 1), u1 = min(max(iu + 1, 0), nr - 1);
    const int64_t v0 = (int64_t)min(max(iv, 0), nc - 1) * nr, v1 = (int64_t)min(max(iv + 1, 0), nc - 1) * nr;
    const float a = __ldg(yp + u0 + v0), b = __ldg(yp + u1 + v0);
    const float c = __ldg(yp + u0 + v1), d = __ldg(yp + u1 + v1);
    const float e0 = fmaf(au, b - a, a), e1 = fmaf(au, d - c, c);
    return fmaf(av, e1 - e0, e0);
}

constexpr int kCtZ = 8;  // voxels along z per thread (the reference's NVOXELS)

// Voxel-driven CT backprojection; thread = (x, y, run of kCtZ voxels in z).
template <bool SENS>
__global__ void k_interp_ct_bp(Grid g, const BddProj *__restrict__ pj, int nr, int nc,
                                                      int64_t nproj, float kerroin, const float *__restrict__ y,
                                                      float *__restrict__ img, float *__restrict__ sens) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int kz0 = blockIdx.z * kCtZ;
    if (i >= g.nx || j >= g.ny || kz0 >= g.nz) return;
    const int nzt = min(kCtZ, g.nz - kz0);
    const float qx = fmaf((float)i, g.dx, g.bx + 0.5f * g.dx);
    const float qy = fmaf((float)j, g.dy, g.by + 0.5f * g.dy);
    const float qz0 = fmaf((float)kz0, g.dz, g.bz + 0.5f * g.dz);
    const float fnr = (float)nr, fnc = (float)nc;
    float temp[kCtZ], wsum[kCtZ];
#pragma unroll
    for (int t = 0; t < kCtZ; ++t) {
        temp[t] = 0.f;
        wsum[t] = 0.f;
    }
    for (int64_t p = 0; p < nproj; ++p) {
        const BddProj P = pj[p];
        const float nu0 = fmaf(P.au[0], qx, fmaf(P.au[1], qy, fmaf(P.au[2], qz0, P.au0)));
        const float nv0 = fmaf(P.av[0], qx, fmaf(P.av[1], qy, fmaf(P.av[2], qz0, P.av0)));
        const float de0 = fmaf(P.c[0], qx, fmaf(P.c[1], qy, fmaf(P.c[2], qz0, 1.f)));
        const float su = P.au[2] * g.dz, sv = P.av[2] * g.dz, sd = P.c[2] * g.dz;
        const float vx = qx - P.s[0], vy = qy - P.s[1];
        const float axy = fmaf(vx, vx, vy * vy);
        const float *yp = y + p * (int64_t)nr * nc;
#pragma unroll
        for (int t = 0; t < kCtZ; ++t) {
            if (t < nzt) {
                const float ft = (float)t;
                const float inv = 1.f / fmaf(ft, sd, de0);
                const float u = fmaf(ft, su, nu0) * inv, v = fmaf(ft, sv, nv0) * inv;
                if (u >= 0.f && u <= fnr && v >= 0.f && v <= fnc) {
                    const float yv = bilinear(yp, nr, nc, u - 0.5f, v - 0.5f);
                    if (yv != 0.f) {
                        const float vz = fmaf(ft, g.dz, qz0) - P.s[2];
                        const float tt = P.k * inv;
                        const float weight = sqrtf(fmaf(vz, vz, axy)) * (tt * tt * tt) * kerroin;
                        temp[t] = fmaf(yv, weight, temp[t]);
                        if (SENS) wsum[t] += weight;
                    }
                }
            }
        }
    }
    int64_t n = i + (int64_t)j * g.nx + (int64_t)kz0 * g.nx * g.ny;
#pragma unroll
    for (int t = 0; t < kCtZ; ++t) {
        if (t < nzt) {
            img[n] = temp[t];
            if (SENS) sens[n] = wsum[t];
        }
        n += (int64_t)g.nx * g.ny;
    }
}

#define OMB_NB_CASES(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

int interp_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, float dL, const float *img,
                   const __nv_bfloat16 *img16, float *y, const Tuning &tn, cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    const unsigned grid = grid_for(rs.m_size, tn.siddon_blocks_per_sm);
    switch (tof.nbins) {
#define X(n)                                                                                    \
    case n:                                                                                     \
        if (img16)                                                                              \
            k_interp_fp<n, __nv_bfloat16><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, dL, img16, y);  \
        else                                                                                    \
            k_interp_fp<n, float><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, dL, img, y);            \
        break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("type-4 forward launch");
    return OMB_OK;
}

template <int NB>
static void bp_launch4(unsigned grid, const Grid &g, const RaySet &rs, const Tof &tof, float gf, float dL,
                       const float *y, float *img, float *sens, unsigned long long *acc, unsigned long long *acc_s,
                       cudaStream_t st) {
    if (acc) {
        if (acc_s)
            k_interp_bp<NB, true, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, dL, y, img, sens, acc, acc_s);
        else
            k_interp_bp<NB, false, true><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, dL, y, img, sens, acc, acc_s);
    } else if (sens) {
        k_interp_bp<NB, true, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, dL, y, img, sens, acc, acc_s);
    } else {
        k_interp_bp<NB, false, false><<<grid, kBlock, 0, st>>>(g, rs, tof, gf, dL, y, img, sens, acc, acc_s);
    }
}

int interp_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, float dL, const float *y, float *img,
                    float *sens, unsigned long long *acc, unsigned long long *acc_s, const Tuning &tn,
                    cudaStream_t st) {
    if (rs.m_size <= 0) return OMB_OK;
    if ((uint64_t)g.nx * g.ny * g.nz >= (1ull << 32))
        return set_error(OMB_ERR_UNSUPPORTED, "type-4 backprojection needs fewer than 2^32 voxels");
    const unsigned grid = grid_for(rs.m_size, tn.siddon_blocks_per_sm);
    switch (tof.nbins) {
#define X(n) case n: bp_launch4<n>(grid, g, rs, tof, gf, dL, y, img, sens, acc, acc_s, st); break;
        OMB_NB_CASES(X)
#undef X
        default:
            return set_error(OMB_ERR_UNSUPPORTED, "TOF bin count above 16 is not built");
    }
    OMB_LAUNCH_CHECK("type-4 backward launch");
    return OMB_OK;
}

int interp_ct_backward(const Grid &g, const BddProj *pj, int nr, int nc, int64_t nproj, float kerroin,
                       const float *y, float *img, float *sens, cudaStream_t st) {
    if (g.nz > 65535 * kCtZ) return set_error(OMB_ERR_UNSUPPORTED, "too many slices");
    dim3 block(32, 8);
    dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kCtZ - 1) / kCtZ);
    if (sens)
        k_interp_ct_bp<true><<<grid, block, 0, st>>>(g, pj, nr, nc, nproj, kerroin, y, img, sens);
    else
        k_interp_ct_bp<false><<<grid, block, 0, st>>>(g, pj, nr, nc, nproj, kerroin, y, img, sens);
    OMB_LAUNCH_CHECK("type-4 CT backward launch");
    return OMB_OK;
}

}  // namespace omb
