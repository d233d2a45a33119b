/*
 * TEST INFRASTRUCTURE ONLY -- a host-side stand-in for the CUDA device
 * environment that OMEGA's kernel sources expect, so that the reference's own
 * kernels (source/opencl/projectorType4.cl, projectorType5.cl, auxKernels.cl,
 * with the CUDA branch of general_opencl_functions.h:544-910) compile
 * unchanged with g++ and run on the CPU as the pinned oracle of projector
 * types 4 and 5, the TV gradient and the PDHG update.  Nothing in the product
 * includes this file.
 *
 * What it supplies (the reference defines everything else itself):
 *   - the CUDA vector types float2/3/4, int2/3/4, uint2/3, long3 and their
 *     make_* constructors (the reference adds the arithmetic operators);
 *   - the device intrinsics the macro layer names (__float2int_rz,
 *     __float2uint_ru/rd/rn, __float2ll_rz, fdividef, __fmaf_rn, __expf,
 *     __frcp_rn, __frsqrt_rn, rsqrtf, __powf, min/max, atomicAdd);
 *   - threadIdx/blockIdx/blockDim/gridDim as thread-local variables that a
 *     driver sets before calling a kernel function once per work item;
 *   - texture objects and tex3D/tex2D with the fetch rules of the CUDA C
 *     Programming Guide ("Texture Fetching"): normalized or unnormalized
 *     coordinates, clamp-to-edge addressing, nearest-point or linear
 *     filtering (x_B = x - 0.5, i = floor(x_B), alpha = frac(x_B)).  Linear
 *     weights are exact by default; frac_bits = 8 rounds them to the guide's
 *     9-bit fixed-point format with 8 fractional bits (round to nearest --
 *     the guide does not state the rounding), which is what the reference's
 *     GPU path computes with.
 *
 * Precision: OMB_REAL is the arithmetic type of the supplied types and
 * functions.  With OMB_REAL = double the including file also maps the
 * keyword `float` to double after this header (ref_cl_wrap.cpp does), so the
 * reference's kernels run in FP64 end to end; the single-precision libm names
 * they call (sqrtf, expf, floorf, ...) are routed to overloads that keep the
 * argument's type.
 */
#ifndef OMB_CL_HOST_SHIM_H
#define OMB_CL_HOST_SHIM_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include <type_traits>

#ifndef OMB_REAL
#define OMB_REAL float
#endif
typedef OMB_REAL omb_real;

/* ---- vector types -------------------------------------------------------- */
struct float2 { omb_real x, y; };
struct float3 { omb_real x, y, z; };
struct float4 { omb_real x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
struct uint2 { unsigned int x, y; };
struct uint3 { unsigned int x, y, z; };
struct long3 { long long x, y, z; };

static inline float2 make_float2(omb_real x, omb_real y) { float2 r = {x, y}; return r; }
static inline float3 make_float3(omb_real x, omb_real y, omb_real z) { float3 r = {x, y, z}; return r; }
static inline float4 make_float4(omb_real x, omb_real y, omb_real z, omb_real w) {
    float4 r = {x, y, z, w}; return r;
}
static inline int2 make_int2(int x, int y) { int2 r = {x, y}; return r; }
static inline int3 make_int3(int x, int y, int z) { int3 r = {x, y, z}; return r; }
static inline int4 make_int4(int x, int y, int z, int w) { int4 r = {x, y, z, w}; return r; }
static inline uint2 make_uint2(unsigned int x, unsigned int y) { uint2 r = {x, y}; return r; }
static inline uint3 make_uint3(unsigned int x, unsigned int y, unsigned int z) { uint3 r = {x, y, z}; return r; }
static inline long3 make_long3(long long x, long long y, long long z) { long3 r = {x, y, z}; return r; }

/* ---- execution-space keywords ------------------------------------------- */
#define __device__
#define __host__
#define __global__
#define __shared__
#define __forceinline__ inline
#define __restrict__
static inline void __syncthreads(void) {}

/* Work-item coordinates: a driver sets blockIdx per work item, with
 * blockDim = 1 and threadIdx = 0, so GID0 = blockIdx.x and so on. */
static thread_local uint3 threadIdx = {0, 0, 0};
static thread_local uint3 blockIdx = {0, 0, 0};
static thread_local uint3 blockDim = {1, 1, 1};
static thread_local uint3 gridDim = {1, 1, 1};

/* ---- scalar intrinsics, kept in the argument's precision ----------------- */
template <class T> static inline T omb_sqrt(T x) { return (T)sqrt((double)x); }
static inline float omb_sqrt(float x) { return sqrtf(x); }
template <class T> static inline T omb_exp(T x) { return (T)exp((double)x); }
static inline float omb_exp(float x) { return expf(x); }
template <class T> static inline T omb_log(T x) { return (T)log((double)x); }
static inline float omb_log(float x) { return logf(x); }
template <class T> static inline T omb_floor(T x) { return (T)floor((double)x); }
static inline float omb_floor(float x) { return floorf(x); }
template <class T> static inline T omb_ceil(T x) { return (T)ceil((double)x); }
static inline float omb_ceil(float x) { return ceilf(x); }
template <class T> static inline T omb_sin(T x) { return (T)sin((double)x); }
static inline float omb_sin(float x) { return sinf(x); }
template <class T> static inline T omb_cos(T x) { return (T)cos((double)x); }
static inline float omb_cos(float x) { return cosf(x); }
template <class T> static inline T omb_acos(T x) { return (T)acos((double)x); }
static inline float omb_acos(float x) { return acosf(x); }
template <class A, class B> static inline typename std::common_type<A, B>::type omb_atan2(A y, B x) {
    typedef typename std::common_type<A, B>::type R;
    return (R)atan2((double)y, (double)x);
}
static inline float omb_atan2(float y, float x) { return atan2f(y, x); }
template <class A, class B> static inline typename std::common_type<A, B>::type omb_pow(A a, B b) {
    typedef typename std::common_type<A, B>::type R;
    return (R)pow((double)a, (double)b);
}
static inline float omb_pow(float a, float b) { return powf(a, b); }
template <class T> static inline T omb_fabs(T x) { return x < (T)0 ? -x : x; }

#define sqrtf(x) omb_sqrt(x)
#define expf(x) omb_exp(x)
#define logf(x) omb_log(x)
#define floorf(x) omb_floor(x)
#define ceilf(x) omb_ceil(x)
#define sinf(x) omb_sin(x)
#define cosf(x) omb_cos(x)
#define acosf(x) omb_acos(x)
#define atan2f(y, x) omb_atan2(y, x)
#define powf(a, b) omb_pow(a, b)
#define fabsf(x) omb_fabs(x)

/* glibc declares its own internal __expf, __logf, __powf, ... so the CUDA
 * fast-math names are macros rather than overloads. */
#define __expf(x) omb_exp(x)
#define __logf(x) omb_log(x)
#define __sinf(x) omb_sin(x)
#define __cosf(x) omb_cos(x)
#define __powf(a, b) omb_pow(a, b)
template <class T> static inline T rsqrtf(T x) { return (T)1 / omb_sqrt(x); }
template <class T> static inline T __frsqrt_rn(T x) { return (T)1 / omb_sqrt(x); }
template <class T> static inline T __frcp_rn(T x) { return (T)1 / x; }
template <class A, class B> static inline typename std::common_type<A, B>::type fdividef(A a, B b) { return a / b; }
template <class A, class B, class C> static inline typename std::common_type<A, B, C>::type __fmaf_rn(A a, B b, C c) {
    typedef typename std::common_type<A, B, C>::type R;
    return (R)fma((double)a, (double)b, (double)c);
}
static inline float __fmaf_rn(float a, float b, float c) { return fmaf(a, b, c); }
template <class T> static inline int __float2int_rz(T x) { return (int)x; }
template <class T> static inline unsigned int __float2uint_ru(T x) { return (unsigned int)omb_ceil(x); }
template <class T> static inline unsigned int __float2uint_rd(T x) { return (unsigned int)omb_floor(x); }
template <class T> static inline unsigned int __float2uint_rn(T x) { return (unsigned int)nearbyint((double)x); }
template <class T> static inline long long __float2ll_rz(T x) { return (long long)x; }

template <class A, class B> static inline typename std::common_type<A, B>::type min(A a, B b) {
    typedef typename std::common_type<A, B>::type R;
    return (R)a < (R)b ? (R)a : (R)b;
}
template <class A, class B> static inline typename std::common_type<A, B>::type max(A a, B b) {
    typedef typename std::common_type<A, B>::type R;
    return (R)a > (R)b ? (R)a : (R)b;
}

/* Atomic adds: the drivers run every scattering kernel on one host thread,
 * so a plain read-modify-write is the atomic update. */
template <class T, class V> static inline T atomicAdd(T *p, V v) {
    T old = *p;
    *p = (T)(old + (T)v);
    return old;
}

/* ---- textures ------------------------------------------------------------ */
typedef struct omb_tex {
    const omb_real *data; /* width fastest, then height, then depth */
    int w, h, d;
    int linear;           /* 1: linear filtering, 0: nearest point */
    int normalized;       /* 1: coordinates in [0, 1] per axis */
    int frac_bits;        /* 0: exact linear weights; 8: 8-bit fractional weights */
} omb_tex;
typedef const omb_tex *cudaTextureObject_t;

static inline int omb_clampi(long long i, int n) {
    return i < 0 ? 0 : (i >= n ? n - 1 : (int)i);
}

static inline omb_real omb_tex_weight(const omb_tex *t, omb_real a) {
    if (t->frac_bits <= 0) return a;
    const double s = (double)(1 << t->frac_bits);
    return (omb_real)(nearbyint((double)a * s) / s);
}

static inline omb_real omb_texel(const omb_tex *t, long long i, long long j, long long k) {
    const int ii = omb_clampi(i, t->w), jj = omb_clampi(j, t->h), kk = omb_clampi(k, t->d);
    return t->data[((size_t)kk * (size_t)t->h + (size_t)jj) * (size_t)t->w + (size_t)ii];
}

static inline omb_real omb_tex_fetch3(const omb_tex *t, omb_real x, omb_real y, omb_real z) {
    if (t->normalized) {
        x *= (omb_real)t->w;
        y *= (omb_real)t->h;
        z *= (omb_real)t->d;
    }
    if (!t->linear)
        return omb_texel(t, (long long)omb_floor(x), (long long)omb_floor(y), (long long)omb_floor(z));
    const omb_real xb = x - (omb_real)0.5, yb = y - (omb_real)0.5, zb = z - (omb_real)0.5;
    const omb_real fx = omb_floor(xb), fy = omb_floor(yb), fz = omb_floor(zb);
    const long long i = (long long)fx, j = (long long)fy, k = (long long)fz;
    const omb_real a = omb_tex_weight(t, xb - fx), b = omb_tex_weight(t, yb - fy), c = omb_tex_weight(t, zb - fz);
    const omb_real one = (omb_real)1;
    return (one - a) * (one - b) * (one - c) * omb_texel(t, i, j, k) +
           a * (one - b) * (one - c) * omb_texel(t, i + 1, j, k) +
           (one - a) * b * (one - c) * omb_texel(t, i, j + 1, k) +
           a * b * (one - c) * omb_texel(t, i + 1, j + 1, k) +
           (one - a) * (one - b) * c * omb_texel(t, i, j, k + 1) +
           a * (one - b) * c * omb_texel(t, i + 1, j, k + 1) +
           (one - a) * b * c * omb_texel(t, i, j + 1, k + 1) +
           a * b * c * omb_texel(t, i + 1, j + 1, k + 1);
}

template <class T> static inline T tex3D(cudaTextureObject_t t, omb_real x, omb_real y, omb_real z) {
    return (T)omb_tex_fetch3(t, x, y, z);
}
template <class T> static inline T tex2D(cudaTextureObject_t t, omb_real x, omb_real y) {
    return (T)omb_tex_fetch3(t, x, y, t->normalized ? (omb_real)0.5 / (omb_real)t->d : (omb_real)0);
}

#endif /* OMB_CL_HOST_SHIM_H */
