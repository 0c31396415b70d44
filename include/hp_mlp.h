/*
 * hp_mlp.h — the learned correction of the Jacobi preconditioner (C-ABI).
 *
 * No counterpart in the reference: the reference's diagonal preconditioner
 * (tri_hp/ins/setup_preconditioner.cpp:9-221, cd/setup_preconditioner.cpp:6-97)
 * uses a hand-tuned formula ("heuristically tuned", ins :170). Here a small
 * multilayer perceptron maps element-local features to a log-scale s_t applied
 * as tprcn(t,:) *= exp(clamp(s_t)) before the scatter to vprcn/sprcn, i.e. a
 * per-element correction of the Jacobi diagonal block and of the local
 * pseudo-time step. s_t = 0 everywhere is the plain method, the fallback.
 *
 * Network: affine layers with ReLU between them and a linear output, widths
 * <= 64, at most 6 layers; inputs standardised by (x - mean) / std. BF16
 * parameters and activations, FP32 accumulation, in hand-written CUDA
 * kernels for inference and training (masked MSE, Adam). All device pointers.
 */
#ifndef HP_MLP_H
#define HP_MLP_H

#include "hp_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hp_mlp hp_mlp;

/* nlayers affine layers, widths[0..nlayers] (inputs ... outputs); deterministic
 * He-uniform initialisation from `seed`. */
int hp_mlp_create(int nlayers, const int *widths, unsigned long long seed, hp_mlp **out);
int hp_mlp_destroy(hp_mlp *net);
int hp_mlp_nparams(const hp_mlp *net);
int hp_mlp_dims(const hp_mlp *net, int *nin, int *nout);
/* input standardisation (host arrays of widths[0] floats) */
int hp_mlp_set_norm(hp_mlp *net, const float *mean, const float *stdv);
/* FP32 master parameters to / from host: [W0 b0 W1 b1 ...], W_l row-major [out][in] */
int hp_mlp_get_params(const hp_mlp *net, float *host);
int hp_mlp_set_params(hp_mlp *net, const float *host);
/* y[n][out] = net(x[n][in]) on `stream` (no synchronisation). */
int hp_mlp_forward(hp_mlp *net, const float *d_x, int n, float *d_y, void *stream);
/* Gradient of 0.5/n sum_s sum_o mask_o (y_so - t_so)^2 to host (nparams floats)
 * and the loss to *loss, without updating; d_mask has widths[nlayers] floats. */
int hp_mlp_grad(hp_mlp *net, const float *d_x, const float *d_t, const float *d_mask, int n, float *host_grad,
                float *loss);
/* One Adam step (beta 0.9 / 0.999) on the same loss; *loss is the loss before it. */
int hp_mlp_train_step(hp_mlp *net, const float *d_x, const float *d_t, const float *d_mask, int n, float lr,
                      float *loss);
const char *hp_mlp_last_error(void);

/* Element features for the network (17 per element, FP32, device array
 * [ntri][17]): for variables n = 0..2 (zero where n >= NV) the mean and spread
 * of the three vertex values and the RMS of the side and of the interior
 * coefficients (12 state moments); log(area/2), log(longest edge), aspect
 * (longest edge^2 / area), log(1 + cell Peclet number) (4 metric terms); p/8. */
#define HP_NFEAT 17
int hp_gpu_elem_features(hp_gpu_ctx *ctx, float *d_feat);

/* Per-element residual measure: sum of squares of the element's own
 * coefficients of the current residual (vertex, side and interior), written to
 * d_out[ntri] (device). */
int hp_gpu_elem_resnorm(hp_gpu_ctx *ctx, double *d_out);

/* Per-element log-scales of the preconditioner from a device array
 * d_logscale[ntri][ld] (variable n uses column min(n, ld-1)), clamped to
 * [-clampv, clampv]; NULL restores the plain preconditioner. The array must stay
 * valid until replaced. Takes effect at the next setup_preconditioner(). */
int hp_gpu_set_prcn_scale(hp_gpu_ctx *ctx, const float *d_logscale, int ld, float clampv);

/* Attaches a trained network: every setup_preconditioner() then evaluates the
 * element features at the current state and the network on the GPU and applies
 * its outputs as the log-scales above. net == NULL detaches it. */
int hp_gpu_set_prcn_net(hp_gpu_ctx *ctx, hp_mlp *net, float clampv);

#ifdef __cplusplus
}
#endif

#endif
