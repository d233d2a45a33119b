// Internal launchers shared between the kernel files and the C-ABI layer.
#pragma once

#include "common.cuh"

namespace omb {

int siddon_forward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, cudaStream_t st);
int siddon_backward(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const Frames &fr, float *sens,
                    cudaStream_t st);
int siddon_backward_fixed(const Grid &g, const RaySet &rs, const Tof &tof, float gf, const float *y,
                          unsigned long long *acc, unsigned long long *acc_sens, cudaStream_t st);
int siddon_count(const Grid &g, const RaySet &rs, const Tof &tof, unsigned long long *total, cudaStream_t st);
int fixed_to_float(const unsigned long long *acc, float *out, int64_t n, cudaStream_t st);

// Elementwise steps of the subset updates.
int osem_ratio(const float *y, float *fp, int64_t n, float epps, cudaStream_t st);
int em_update(float *img, const float *sens, const float *rhs, int64_t n, float epps, cudaStream_t st);
int clamp_min(float *x, int64_t n, float lo, cudaStream_t st);
size_t reduce_workspace_bytes(int64_t n);
int loglik(const float *y, const float *fp, int64_t n, float epps, double *out_host, void *work,
           cudaStream_t st);

}  // namespace omb
