/*
 * wr_net.h - kernels of the learned warm-start network (no counterpart in the
 * reference).  A small 3-D convolutional encoder-decoder predicts a coarse
 * displacement field from a template / moving pair; the registration takes it
 * through the reference's warm-start channel option["motion"]
 * (src/wholistic_registration/utils/calFlow3d_Wei_v1.py:362-377).
 *
 * Tensors are channels-last bfloat16 [n][z][y][x][c] on the device, channel
 * counts multiples of 16.  A 3x3x3 convolution (padding 1, stride 1 or 2) may
 * read the virtual concatenation of two sources: source 1 (c1 channels,
 * optionally at half resolution and read nearest-upsampled) and source 2
 * (c2 channels, the input grid).  Weights are float32 masters
 * [27][cout_p][cin] (cout_p = cout rounded up to 16, padding rows zero) with
 * bfloat16 copies for the forward pass and transposed [27][cin][cout_p] for
 * the data gradient.  Same return codes as wr_b200.h.
 */
#ifndef WR_NET_H
#define WR_NET_H

#include <stddef.h>
#include <stdint.h>

#include "wr_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t n;              /* batch */
  int32_t oz, oy, ox;     /* output grid */
  int32_t iz, iy, ix;     /* input grid of source 2 (or of source 1 when up1 = 0) */
  int32_t stride;         /* 1 or 2 */
  int32_t c1, c2;         /* channels of source 1 / source 2 (c2 = 0: one source) */
  int32_t up1;            /* source 1 is half resolution (decoder skip join) */
  int32_t cout;           /* output channels (<= 64) */
  int32_t act;            /* 1: LeakyReLU(0.1) */
} WrConvGeom;

/* Message of the last failed network call on this thread. */
WR_API const char* wr_net_last_error(void);

/* The convolutions run on the tcgen05 tensor cores with TMEM accumulators and
   bounded waits: *flag = 1 when a launch on the current device gave up
   waiting for its tensor-core work since the last call (the flag is then
   cleared).  Synchronises the device. */
WR_API int wr_net_tc_error(int* flag);

/* y = act(conv(x) + bias): bf16 output [n][o][cout], or float32 when y32 != NULL. */
WR_API int wr_net_conv3d_fwd(const WrConvGeom* g, const void* x1, const void* x2, const void* w_bf16,
                             const float* bias, void* y, float* y32, void* stream);

/* Gradient of the (virtual concatenated) input: dxv float32 [n][i][cin] from
   dy bf16 [n][o][cout_p] and the transposed bf16 weights. */
WR_API int wr_net_conv3d_dgrad(const WrConvGeom* g, const void* dy, const void* wt_bf16, float* dxv, void* stream);

/* Weight and bias gradients, accumulated (+=) into float32 dw [27][cout_p][cin] and db [cout]. */
WR_API int wr_net_conv3d_wgrad(const WrConvGeom* g, const void* x1, const void* x2, const void* dy, float* dw,
                               float* db, void* stream);

/* dpre = grad * LeakyReLU'(y) (act = 1) or grad (act = 0), bf16 padded to cout_p channels. */
WR_API int wr_net_act_backward(const float* grad, const void* y, int act, void* dpre, long long nvox, int cout,
                               void* stream);

/* Scatter dxv into the sources' float32 gradients (+=); source 1's part is
   summed over its 2x2x2 fine voxels when up1 = 1.  Either output may be NULL. */
WR_API int wr_net_split_grad(const WrConvGeom* g, const float* dxv, float* g1, float* g2, void* stream);

/* One Adam step (bias-corrected, L2 decay added to the gradient). */
WR_API int wr_net_adam(float* w, const float* gw, float* m, float* v, long long n, float lr, float b1, float b2,
                       float eps, int step, float decay, void* stream);

/* float32 master weights -> bf16 forward weights and (if wt != NULL) transposed bf16 weights. */
WR_API int wr_net_weights_to_bf16(const float* w, void* wf, void* wt, int cout, int cin, void* stream);

/* Loss l2 * mean|pred - target|^2 + res * mean(mov(p + pred) - tmpl)^2 on the
   network grid (flow in full-resolution voxels, x / y divided by `scale` on
   the grid); writes d loss / d pred and adds the loss to *loss. */
WR_API int wr_net_flow_loss(const float* pred, const float* target, const float* tmpl, const float* mov,
                            float* grad, double* loss, int n, int nz, int ny, int nx, float scale, float l2,
                            float res, void* stream);

/* Network input from a (z, y, x) template / moving pair (uint16 or float32):
   factor x factor mean pooling in x and y, divided by the template's mean
   (computed into *mean_scratch, one device double); x0 bf16 [z][y/f][x/f][16]
   with channels 0 / 1 = template / moving; t4, m4 (nullable) float32 copies. */
WR_API int wr_net_prepare_input(const WrVolume* tmpl, const WrVolume* mov, int factor, double* mean_scratch,
                                void* x0, float* t4, float* m4, void* stream);

/* Adds sum((a - b)^2) and the voxel count over voxels with excl == 0 (or all
   when excl is NULL) to out2[0], out2[1]; a float32, b uint16 or float32.
   Used to compare a warm-started registration's residual with the plain
   method's. */
WR_API int wr_net_masked_sse(const float* a, const WrVolume* b, const uint8_t* excl, double* out2, void* stream);

/* Flow (z, y, x, 3) -> factor x factor mean pooling in x and y. */
WR_API int wr_net_pool_flow(const float* flow, int nz, int ny, int nx, int factor, float* out, void* stream);

/* Coarse flow (z, y/f, x/f, 3) -> (z, y, x, 3), bilinear in x and y. */
WR_API int wr_net_upsample_flow(const float* fq, int nz, int ny, int nx, int factor, float* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WR_NET_H */
