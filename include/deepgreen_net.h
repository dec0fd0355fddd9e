/* deepgreen_net.h -- C ABI of the learned coarse-grid correction.
 *
 * The reference solver has no learned component; this interface is an
 * addition.  It holds a small 3-D convolutional network that maps a
 * 2x-coarsened Euler state (after one plain coarse step) to a correction of
 * its conserved variables, trained on pairs the solver itself generates.
 *
 * Network: 4 layers of 3x3x3 "valid" convolutions, inputs -> hidden ->
 * hidden -> hidden -> outputs, GELU after layers 1-3 (tanh form,
 * x/2 (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3)))), linear last layer.  Weights and activations BF16, accumulation FP32 on the tensor
 * cores; master weights, gradients and Adam moments FP32.  Channels are padded
 * to DG_NET_IO_CHANNELS at the input and output (padding channels are zero).
 *
 * Device tensors are channels-last, [n][x][y][z][C] with C = 16, z fastest
 * (BF16 inputs, FP32 outputs and targets).  A forward pass over an input of
 * extents (X, Y, Z) produces (X-8, Y-8, Z-8).
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

/* Inference.  feat: device BF16 [n][x][y][z][16] (16-byte aligned); out:
 * device FP32 [n][x-8][y-8][z-8][16] (32-byte aligned).  Asynchronous on the
 * network's stream. */
int32_t dg_net_forward(dg_net *net, const void *feat, int32_t n, int32_t x, int32_t y, int32_t z, float *out);

/* One forward + backward pass.  feat: device BF16 [n][x][y][z][16]; target:
 * device FP32 [n][x-8][y-8][z-8][16] (first `outputs` channels used).  Loss
 * = mean over positions and real outputs of (out - target)^2, returned in
 * *loss (synchronises).  Gradients are kept in the network (replacing the
 * previous ones) for dg_net_get_grad / dg_net_adam_step. */
int32_t dg_net_forward_backward(dg_net *net, const void *feat, const float *target, int32_t n, int32_t x,
                                int32_t y, int32_t z, double *loss);

/* The same in flux form, for a network with 15 outputs: output channel
 * 5 d + c is the flux of conserved field c through the upper face of a cell
 * along axis d (x, y, z), and the correction of cell t is the divergence
 * dU_c(t) = sum_d F_{d,c}(t) - F_{d,c}(t - e_d) -- exactly conservative, and
 * zero wherever the fluxes are uniform.  Cubic crops: feat of extents x^3,
 * network output (x-8)^3, target FP32 [n][x-9][x-9][x-9][16] (first 5
 * channels: the corrections of the cells whose lower faces the output also
 * covers).  Loss = mean over cells and the 5 fields of w_b (dU - target)^2,
 * w_b = 1, or with `balance` = mean target power of the batch / (target power
 * of entry b + 0.01 x that mean): every crop counts alike, whether its
 * corrections are large (shear layers) or small (smooth flow). */
int32_t dg_net_forward_backward_flux(dg_net *net, const void *feat, const float *target, int32_t n, int32_t x,
                                     int32_t y, int32_t z, int32_t balance, double *loss);

/* Adam update of all parameters from the stored gradients (bias-corrected,
 * step counter kept by the network). */
int32_t dg_net_adam_step(dg_net *net, float lr, float beta1, float beta2, float eps);

/* Copy of an intermediate tensor of the last forward_backward, for tests:
 * which = 0 activation (after GELU, BF16 bits), 1 pre-activation (BF16
 * bits), 2 network output (FP32), 3 gradient w.r.t. the pre-activation (BF16
 * bits, unpadded), channels-last [n][x][y][z][C].  Layer 0..3; host
 * buffer sized by the caller. */
int32_t dg_net_get_tensor(dg_net *net, int32_t layer, int32_t which, void *host, uint64_t bytes);

/* ---- Learned coarse step -------------------------------------------------
 *
 * The network corrects a coarse grid after each plain step.  Its 14 input
 * channels per cell, from the conserved densities before (U0) and after (U1)
 * the plain step (density = per-cell total / ds^3):
 *   0 rho1, 1-3 (rho v)1, 4 E1,  5-9 U1 - U0 (same order),
 *   10-12 v1 = (rho v)1 / rho1,  13 p1 = (gamma-1)(E1 - |(rho v)1|^2 / (2 rho1)),
 * each normalised as (raw - in_mean[c]) * in_inv_std[c] (channels 14, 15 are
 * zero).  The network has 15 outputs, face fluxes in flux form (see
 * dg_net_forward_backward_flux); their divergence is the correction of
 * conserved density c in units of out_std[c].  Grids must be cubic and
 * periodic: the network's 4-cell halo and the divergence wrap around.
 *
 * "State packs" are dense device copies of a grid's conserved state: 5
 * fields (mass, mom_x, mom_y, mom_z, energy) of (n+4)^3 FP32 values each, C
 * order with ghosts, consecutive -- what dg_get_conserved_device writes when
 * given pointers 1, 2, ... fields apart. */
#define DG_LEARNED_INPUTS 14
#define DG_LEARNED_OUTPUTS 15

typedef struct dg_learned_norm {
    float in_mean[16];
    float in_inv_std[16];
    float out_std[16];
} dg_learned_norm;

/* coarse := 2x2x2 sums of fine's per-cell totals over the interior (fine
 * interior extents twice the coarse ones, both FP32); ghosts and the next dt
 * of the coarse grid follow as after dg_set_conserved.  Synchronises. */
int32_t dg_coarsen(dg_ctx *fine, dg_ctx *coarse);

/* Network inputs of a crop of a periodic cubic grid with n interior cells per
 * axis, from state packs `before` and `after`: ext^3 cells starting at
 * interior cell (ox, oy, oz) (wrapped), written as BF16 [ext][ext][ext][16]
 * to feat.  Asynchronous on `stream` (cudaStream_t or NULL). */
int32_t dg_learned_features(const dg_learned_norm *norm, const float *before, const float *after, int32_t n, double ds,
                            double gamma, int32_t ox, int32_t oy, int32_t oz, int32_t ext, void *feat, void *stream);

/* Training targets: (truth - after) / ds^3 / out_std per field over the ext^3
 * cells starting at (ox, oy, oz), FP32 [ext][ext][ext][16] (channels >= 5
 * zero).  Asynchronous on `stream`. */
int32_t dg_learned_targets(const dg_learned_norm *norm, const float *after, const float *truth, int32_t n, double ds,
                           int32_t ox, int32_t oy, int32_t oz, int32_t ext, float *out, void *stream);

typedef struct dg_corrector dg_corrector;

typedef struct dg_learned_stats {
    uint64_t steps;           /* corrected steps attempted */
    uint64_t fallback_steps;  /* steps that kept the plain coarse state everywhere */
    uint64_t masked_cells;    /* cells that kept their plain value (rho or p would not stay positive) */
    uint64_t cells;           /* cells examined: steps x n^3 */
    double max_drift;         /* largest |sum(U' - U)| / sum|U| over fields, accepted steps */
    double last_drift;        /* the same for the latest step, kept or not */
    uint64_t violations;      /* cells that lost positivity after the mean removal (each rejects its step) */
} dg_learned_stats;

/* A corrector couples a coarse FP32 context (cubic, periodic, n a multiple of
 * 4 and at most 1024 cells per axis) and a network
 * (14 inputs, 15 flux outputs).  Each step: one plain step; the network's
 * correction, zero in cells where rho or p of the corrected state would not
 * be positive, minus its mean over the other cells; the whole step falls back
 * to the plain state if a cell still loses positivity or the correction
 * changes a field's total by more than `tolerance` (default 1e-10) of its
 * L1 norm; the next dt comes from the state kept. */
int32_t dg_corrector_create(dg_ctx *coarse, dg_net *net, const dg_learned_norm *norm, dg_corrector **out);
/* The context and the network are not owned: they must outlive every step of
 * the corrector.  Destroying the corrector touches neither, so it may come
 * after them. */
int32_t dg_corrector_destroy(dg_corrector *cor);
int32_t dg_corrector_set_tolerance(dg_corrector *cor, double tolerance);
/* nsteps corrected steps, asynchronous on the context's stream (dg_get_dts
 * and dg_synchronize of the context apply). */
int32_t dg_corrector_step(dg_corrector *cor, int32_t nsteps);
/* Totals since creation; synchronises. */
int32_t dg_corrector_stats(dg_corrector *cor, dg_learned_stats *out);
const char *dg_corrector_last_error(const dg_corrector *cor);

int32_t dg_net_synchronize(dg_net *net);
void *dg_net_get_stream(dg_net *net);
const char *dg_net_last_error(const dg_net *net);

#ifdef __cplusplus
}
#endif

#endif /* DEEPGREEN_NET_H */
