/*
 * omega_b200_unet.h -- C-ABI of the kernels of the learned OSEM warm start:
 * a 3-D U-Net (3x3x3 convolutions, BF16 weights and activations, FP32
 * accumulation) trained and run on the GPU by these kernels.  The reference
 * has no counterpart: OMEGA has no learned component on this path.
 *
 * Layouts: activations channels-last BF16 [B][Z][Y][X][C] (C a multiple of
 * 16); conv weights BF16 [27][Cout][Cin], tap = (dz+1)*9 + (dy+1)*3 + (dx+1);
 * biases, master weights, gradients and optimiser state FP32.  Volumes
 * handed in/out as FP32 Fortran order (x fastest) like the projector images.
 * Status codes and stream conventions as in omega_b200.h.
 */
#ifndef OMEGA_B200_UNET_H
#define OMEGA_B200_UNET_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/*
 * out = conv3x3x3(in, w) + bias, ReLU when relu != 0; with relu_mask != NULL
 * the output is instead multiplied by (relu_mask > 0) (the data gradient of
 * the previous ReLU, used with flipped weights for backpropagation).
 * Built shapes (cin, cout): (16,16) (16,32) (32,32) (32,64) (64,64) (96,32)
 * (48,16) (32,16) (64,32) (32,96) (16,48).  bias may be NULL.
 */
int omb_unet_conv(int32_t cin, int32_t cout, const void *in, const void *w, const float *bias, void *out,
                  const void *relu_mask, int32_t relu, int32_t X, int32_t Y, int32_t Z, int32_t B, void *stream);

/*
 * The same convolution on the 5th-generation tensor cores (tcgen05.mma with
 * the accumulator in tensor memory, 128 voxels x cout per CTA), for the same
 * shapes and arguments as omb_unet_conv.  Its waits on the tensor core are
 * bounded: a wait that gives up skips the output and raises the flag that
 * omb_unet_take_error reads.
 */
int omb_unet_conv_tc(int32_t cin, int32_t cout, const void *in, const void *w, const float *bias, void *out,
                     const void *relu_mask, int32_t relu, int32_t X, int32_t Y, int32_t Z, int32_t B, void *stream);

/* Reads and clears the tensor-core convolutions' timeout flag (synchronises the device). */
int omb_unet_take_error(int32_t *out_host);

/* dw[27][cout][cin] += sum_v dz[v][co] in[v + off(tap)][ci] (FP32; dw must be zeroed by the caller). */
int omb_unet_conv_wgrad(int32_t cin, int32_t cout, const void *in, const void *dz, float *dw, int32_t X, int32_t Y,
                        int32_t Z, int32_t B, void *stream);

/*
 * The same weight gradient on the tensor cores (tcgen05.mma, the voxels as
 * the reduction dimension, 128 rows of (tap, ci) x cout per CTA accumulated in
 * tensor memory, FP32 atomics into dw), for the shapes omb_unet_conv_tc
 * builds.  Its waits are bounded like omb_unet_conv_tc's (flag read by
 * omb_unet_take_error).
 */
int omb_unet_conv_wgrad_tc(int32_t cin, int32_t cout, const void *in, const void *dz, float *dw, int32_t X,
                           int32_t Y, int32_t Z, int32_t B, void *stream);

/* db[c] += sum_v dz[v][c], c in {16, 32, 64}. */
int omb_unet_bias_grad(int32_t c, const void *dz, float *db, int64_t nvox, void *stream);

/* wf[tap][ci][co] = w[26 - tap][co][ci]: the weights of the data-gradient convolution. */
int omb_unet_flip_weights(const void *w, void *wf, int32_t cin, int32_t cout, void *stream);

/* 2x2x2 average pooling of in ([..][Z][Y][X][C]) into out; backward != 0: in is dout, out (din) += dout / 8. */
int omb_unet_avgpool(const void *in, void *out, int32_t X, int32_t Y, int32_t Z, int32_t B, int32_t C,
                     int32_t backward, void *stream);

/* cat = [nearest 2x upsampling of low (cl channels), skip (cs channels)] at full size X x Y x Z. */
int omb_unet_up_concat(const void *low, const void *skip, void *cat, int32_t X, int32_t Y, int32_t Z, int32_t B,
                       int32_t cl, int32_t cs, void *stream);

/* Backward of omb_unet_up_concat: dlow = sum of the 8 children, dskip += its channels of dcat. */
int omb_unet_up_concat_bwd(const void *dcat, void *dlow, void *dskip, int32_t X, int32_t Y, int32_t Z, int32_t B,
                           int32_t cl, int32_t cs, void *stream);

/* d = d * (a > 0) over n BF16 elements. */
int omb_unet_relu_mask(void *d, const void *a, int64_t n, void *stream);

/*
 * Network input [B][Z][Y][X][16]: channel 0 = osem_b * scale[b], channel 1 =
 * sens * sens_scale, the rest 0; slices z >= Zs (padding) are 0.  osem: B
 * FP32 Fortran-order volumes of X*Y*Zs voxels, osem_stride apart.
 */
int omb_unet_make_input(const float *osem, int64_t osem_stride, const float *sens, const float *scale,
                        float sens_scale, void *out, int32_t X, int32_t Y, int32_t Z, int32_t Zs, int32_t B,
                        void *stream);

/* pred[v] = input channel 0 + bias + sum_c w[c] a[v][c] (16 channels), FP32. */
int omb_unet_head_fwd(const void *a, const void *inp, const float *w, const float *bias, float *pred, int64_t nvox,
                      void *stream);

/*
 * Mean squared error against target * tscale[b] over the slices z < Zs,
 * added to *loss (device); da = dL/da masked by (a > 0); dw, db += head
 * gradients (zeroed by the caller).
 */
int omb_unet_head_bwd(const void *a, const float *pred, const float *target, int64_t target_stride,
                      const float *tscale, const float *w, void *da, float *dw, float *db, float *loss, int32_t X,
                      int32_t Y, int32_t Z, int32_t Zs, int32_t B, void *stream);

/* out_b (Fortran order, z < Zs) = max(pred / scale[b], floor_v). */
int omb_unet_head_out(const float *pred, const float *scale, float *out, int64_t out_stride, float floor_v, int32_t X,
                      int32_t Y, int32_t Z, int32_t Zs, int32_t B, void *stream);

/* One Adam step on FP32 master weights p (moments m, v; gradient g); p_bf16 (may be NULL) receives the BF16 copy. */
int omb_unet_adam(float *p, float *m, float *v, const float *g, void *p_bf16, int64_t n, float lr, float beta1,
                  float beta2, int32_t step, float eps, void *stream);

/* b = bf16(a) over n elements. */
int omb_unet_to_bf16(const float *a, void *b, int64_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif
