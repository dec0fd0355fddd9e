/* deepgreen_net.h -- C ABI of the learned coarse-grid correction.
 *
 * The reference solver has no learned component; this interface is an
 * addition.  It holds a small 3-D convolutional network that maps a
 * 2x-coarsened Euler state (after one plain coarse step) to a correction of
 * its conserved variables, trained on pairs the solver itself generates.
 *
 * Network: 4 layers of 3x3x3 "valid" convolutions, inputs -> hidden ->
 * hidden -> hidden -> outputs, GELU (erf form) after layers 1-3, linear last
 * layer.  Weights and activations BF16, accumulation FP32 on the tensor
 * cores; master weights, gradients and Adam moments FP32.  Channels are padded
 * to DG_NET_IO_CHANNELS at the input and output (padding channels are zero).
 *
 * Tensors on the device are channels-last, [n][x][y][z][C], z fastest.  A
 * forward pass over an input of extents (X, Y, Z) produces (X-8, Y-8, Z-8).
 *
 * Layouts of parameters exchanged with the host: weights of layer l as FP32
 * [cout][cin][3][3][3] over the REAL channel counts (the layout of
 * torch.nn.Conv3d on tensors ordered (n, C, x, y, z)), biases [cout].
 *
 * Every function returns DG_OK (0) or a negative DG_ERR_* code from
 * deepgreen.h; dg_net_last_error() describes the last failure.
 */
#ifndef DEEPGREEN_NET_H
#define DEEPGREEN_NET_H

#include <stdint.h>

#include "deepgreen.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DG_NET_IO_CHANNELS 16   /* padded input and output channels */
#define DG_NET_HIDDEN 32        /* hidden channels */
#define DG_NET_LAYERS 4

typedef struct dg_net dg_net;

typedef struct dg_net_info {
    int32_t inputs;     /* real input channels, 1..16 */
    int32_t outputs;    /* real output channels, 1..16 */
    int32_t device;     /* CUDA device ordinal */
    int32_t pad;
    uint64_t seed;      /* weight initialisation */
    double out_scale;   /* initial weights of the last layer are scaled by this */
} dg_net_info;

int32_t dg_net_create(const dg_net_info *info, dg_net **out);
int32_t dg_net_destroy(dg_net *net);

/* Parameters and gradients of layer l (0..3), host FP32, real channels. */
int32_t dg_net_set_layer(dg_net *net, int32_t layer, const float *w, const float *b);
int32_t dg_net_get_layer(dg_net *net, int32_t layer, float *w, float *b);
int32_t dg_net_get_grad(dg_net *net, int32_t layer, float *gw, float *gb);

/* Inference.  feat: device BF16 [n][x][y][z][16]; out: device FP32
 * [n][x-8][y-8][z-8][16].  Asynchronous on the network's stream. */
int32_t dg_net_forward(dg_net *net, const void *feat, int32_t n, int32_t x, int32_t y, int32_t z, float *out);

/* One forward + backward pass.  feat: device BF16 [n][x][y][z][16]; target:
 * device FP32 [n][x-8][y-8][z-8][16] (first `outputs` channels used).  Loss
 * = mean over positions and real outputs of (out - target)^2, returned in
 * *loss (synchronises).  Gradients are kept in the network (replacing the
 * previous ones) for dg_net_get_grad / dg_net_adam_step. */
int32_t dg_net_forward_backward(dg_net *net, const void *feat, const float *target, int32_t n, int32_t x,
                                int32_t y, int32_t z, double *loss);

/* Adam update of all parameters from the stored gradients (bias-corrected,
 * step counter kept by the network). */
int32_t dg_net_adam_step(dg_net *net, float lr, float beta1, float beta2, float eps);

/* Copy of an intermediate tensor of the last forward_backward, for tests:
 * which = 0 activation (after GELU, BF16 bits), 1 pre-activation (BF16
 * bits), 2 network output (FP32), 3 gradient w.r.t. the pre-activation (BF16
 * bits, unpadded).  Layer 0..3; host buffer sized by the caller. */
int32_t dg_net_get_tensor(dg_net *net, int32_t layer, int32_t which, void *host, uint64_t bytes);

int32_t dg_net_synchronize(dg_net *net);
void *dg_net_get_stream(dg_net *net);
const char *dg_net_last_error(const dg_net *net);

#ifdef __cplusplus
}
#endif

#endif /* DEEPGREEN_NET_H */
