/*
 * unet3d.h — C ABI of libunet3d.so: the kernels of the learned warm start, a small
 * 3-D convolutional U-Net that predicts the steady density/velocity field of a
 * channel flow from the body mask, its signed distance and the Reynolds number.
 * No counterpart in the reference (LBM3D_BB starts every run from rest,
 * Initialization.jl:11-70); the network seeds lbm_init_equilibrium (lbm3d.h).
 *
 * Tensors are device arrays in channels-last order, element (n, z, y, x, c) at
 * c + C*(x + W*(y + H*(z + D*n))).  Activations and working weights are BF16,
 * accumulation is FP32 (tensor-core MMA), master weights, gradients and optimiser
 * moments are FP32.  Convolution weights are stored [27 taps][Cout][Cin], tap =
 * (dz+1)*9 + (dy+1)*3 + (dx+1), zero padding of one voxel on every face.
 *
 * Every entry point enqueues on `stream` (a cudaStream_t, NULL = legacy default)
 * and returns 0 or a nonzero status with nn_last_error() describing it.
 * Shape rules: Cin and Cout multiples of 16 (Cout of a forward convolution at
 * most 96), W a multiple of 16, pooled grids need even D, H, W.
 */
#ifndef UNET3D_H
#define UNET3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UNET3D_ABI_VERSION 1

int32_t nn_abi_version(void);
const char* nn_last_error(void);

/* out = act(conv3x3x3(in, w) + bias); act = ReLU when relu != 0.  bias may be NULL. */
int32_t nn_conv3d_fwd(const void* in, const void* w, const float* bias, void* out, int32_t n, int32_t d,
                      int32_t h, int32_t wd, int32_t cin, int32_t cout, int32_t relu, void* stream);
/* Engine of nn_conv3d_fwd (and so of the data gradient): 0 = mma.sync warp tiles
 * (FP32 accumulation in registers); 1 = tcgen05 (128-voxel CTA tiles gathered into
 * shared memory by the threads, FP32 accumulator in tensor memory); 2 = per layer
 * (default: tcgen05 for Cout >= 32, warp tiles for Cout = 16); 3 = tcgen05 with the tiles
 * loaded by TMA (5-D tensor map, zero fill for the halo) where nn_conv_uses_tma says so,
 * else as 1.  Returns the previous engine, or -1 with nn_last_error() for an unknown
 * engine.  Process-wide. */
int32_t nn_set_conv_engine(int32_t engine);
/* 1 when a forward convolution of this shape runs the TMA-fed tcgen05 kernel under the
 * current engine (engine 3, tiles of 128 voxels = whole rows or part of one row, a
 * tensor-map encoder from the driver), 0 when it runs one of the other kernels. */
int32_t nn_conv_uses_tma(int32_t h, int32_t wd, int32_t cin, int32_t cout);
/* Blocking: nonzero (and cleared) when a tcgen05 convolution gave up waiting for its
 * matrix multiply since the last call; its output is then not valid. */
int32_t nn_tc_status(void* stream);
/* Self-test of the bounded tcgen05 pipeline waits (no counterpart in the reference).
 * One block waits on an mbarrier that no MMA commits to, through the same bounded wait
 * the convolution kernels use, with a limit of `polls` polls (1 .. 2^22); the wait gives
 * up, the block sets the error word and returns with nothing in flight, and the call
 * returns the nn_tc_status of that (nonzero, word cleared).  Blocking. */
int32_t nn_wait_selftest(int32_t polls, void* stream);
/* Weights of the data gradient: wt[26 - tap][ci][co] = w[tap][co][ci]; then
 * din = nn_conv3d_fwd(dout, wt, NULL, din, ..., cin = cout, cout = cin, relu = 0). */
int32_t nn_conv3d_flip(const void* w, void* wt, int32_t cin, int32_t cout, void* stream);
/* dw[tap][co][ci] += sum over voxels of dout[v][co] * in[v + off(tap)][ci] (FP32). */
int32_t nn_conv3d_bwd_weight(const void* in, const void* dout, float* dw, int32_t n, int32_t d, int32_t h,
                             int32_t wd, int32_t cin, int32_t cout, void* stream);
/* db[c] += sum over voxels of dout[v][c] (FP32). */
int32_t nn_bias_grad(const void* dout, float* db, int64_t voxels, int32_t c, void* stream);
/* dy *= (y > 0), elementwise over `count` BF16 values (ReLU backward). */
int32_t nn_relu_bwd(void* dy, const void* y, int64_t count, void* stream);
/* 2x2x2 average pooling of a fine grid (d, h, wd) to (d/2, h/2, wd/2). */
int32_t nn_pool2(const void* in, void* out, int32_t n, int32_t d, int32_t h, int32_t wd, int32_t c, void* stream);
/* din (=, or += when accumulate != 0) = dout of the parent / 8. */
int32_t nn_pool2_bwd(const void* dout, void* din, int32_t n, int32_t d, int32_t h, int32_t wd, int32_t c,
                     int32_t accumulate, void* stream);
/* out[.., 0:cu] = nearest 2x upsampling of low, out[.., cu:cu+cs] = skip (fine grid d, h, wd). */
int32_t nn_up2_concat(const void* low, const void* skip, void* out, int32_t n, int32_t d, int32_t h, int32_t wd,
                      int32_t cu, int32_t cs, void* stream);
/* dlow = sum of the 8 children of dcat[.., 0:cu]; dskip = dcat[.., cu:cu+cs] (both assigned). */
int32_t nn_up2_concat_bwd(const void* dcat, void* dlow, void* dskip, int32_t n, int32_t d, int32_t h, int32_t wd,
                          int32_t cu, int32_t cs, void* stream);
/* Masked mean squared error of the first ct channels of out (cpad channels, BF16)
 * against target (ct channels, FP32) over voxels with mask != 0 (per-channel
 * weights cw[ct]): loss[0] += sum cw_c (o - t)^2 / count, dout = d loss / d out
 * (zero elsewhere), count = number of masked voxels (given). */
int32_t nn_mse(const void* out, const float* target, const uint8_t* mask, const float* cw, void* dout,
               double* loss, int64_t voxels, int32_t cpad, int32_t ct, double count, void* stream);
/* Adam with bias correction (step t >= 1) on FP32 master weights w, refreshing the
 * BF16 working copy wb (may be NULL). */
int32_t nn_adam(float* w, const float* g, float* m, float* v, void* wb, int64_t count, float lr, float beta1,
                float beta2, float eps, int32_t t, void* stream);
/* out[0] += sum (a - b)^2 and out[1] += sum a^2 over `count` FP32 values (FP64 sums):
 * the relative change of a field between two checks of a run to steady state. */
int32_t nn_diff_norms(const float* a, const float* b, int64_t count, double* out, void* stream);
/* Network input of one channel case with an ellipsoid body (centre, row-major
 * body->world rotation, semi-axes; lattice units), BF16 (nz, ny, nx, 16): solid mask
 * (the solver's rasterisation), signed distance / 16 clipped to [-1, 4], re_feature,
 * node position x/nx, y/ny, z/nz, zeros. */
int32_t nn_features_ellipsoid(void* out, int32_t nx, int32_t ny, int32_t nz, const double* center,
                              const double* rot, const double* semi, float re_feature, void* stream);
/* out (n, 4, d, h, w), FP32 planar: = (or += when accumulate != 0) weight * the first
 * four channels of the network output y (n, d, h, w, 16), read from its mirror image in
 * y (flip_y) and/or z (flip_z) with the mirrored velocity components (channels 2, 3)
 * negated — the prediction for a reflected input mapped back to the original frame. */
int32_t nn_unpack_fields(const void* y, float* out, int32_t n, int32_t d, int32_t h, int32_t wd, int32_t flip_y,
                         int32_t flip_z, float weight, int32_t accumulate, void* stream);
/* FP32 -> BF16 (round to nearest even) and BF16 -> FP32. */
int32_t nn_to_bf16(const float* x, void* y, int64_t count, void* stream);
int32_t nn_from_bf16(const void* x, float* y, int64_t count, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* UNET3D_H */
