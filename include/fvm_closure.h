/* C ABI of the learned flux-correction closure in libfvm_b200.
 *
 * The reference (nathanzimniak/multiphysics-fvm) has no learned part: these
 * entry points are new.  They sit on the coarse-grid MUSCL interface fluxes
 * of the navier_stokes residual (src/physics/navier_stokes.py:588-711, the
 * face fluxes of :627-660) and on the Runge-Kutta stage update
 * (src/numerics/time_integrators.py:106-159), which is where a corrected flux
 * enters the reference's algorithm; everything else is unchanged.
 *
 * Network: periodic 3x3x3 convolutions 16 -> 32 -> 32 -> 16 channels with
 * ReLU after the first two, BF16 weights and activations, FP32 accumulation
 * on the tensor cores.  Input channels 0..4 are the normalised primitive
 * variables (rho, v1, v2, v3, p) of a cell; output channel a*5+q (a = face
 * axis, q = conserved variable) is the correction to the flux of q through
 * the +x_a face of the cell, in units of out_scale[q].  Weights are exchanged
 * as float32 W[27][cout][cin] (tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)) and
 * b[cout]; layer dims (cout, cin) are (32, 16), (32, 32), (16, 32).
 *
 * Dense device arrays ("dense") are float32 [q][k][j][i] with i (x1) fastest.
 * All calls return 0 or a negative FVM_E_* code from fvm.h; fvm_last_error()
 * gives the message.  Device pointers passed in must stay valid until the call
 * returns; calls that take one synchronise before returning.
 */
#ifndef FVM_CLOSURE_H
#define FVM_CLOSURE_H

#include "fvm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fvm_closure fvm_closure;

/* Buffers reachable through fvm_closure_buffer (layouts [pos][channels]). */
#define FVM_CB_X0 0  /* bf16 x16: features */
#define FVM_CB_A1 1  /* bf16 x32: layer-1 activation */
#define FVM_CB_A2 2  /* bf16 x32: layer-2 activation */
#define FVM_CB_Z3 3  /* f32  x16: network output (face corrections / out_scale) */
#define FVM_CB_G3 4  /* bf16 x16: dLoss/dZ3 */
#define FVM_CB_G2 5  /* bf16 x32: dLoss/d(layer-2 pre-activation) */
#define FVM_CB_G1 6  /* bf16 x32: dLoss/d(layer-1 pre-activation) */
#define FVM_CB_E 7   /* f32 dense [5][pos]: predicted minus target defect */

/* Network and workspace for one periodic grid n1 x n2 x n3 (n1 % 16 == 0,
 * n2 % 16 == 0, n3 >= 1).  Weights He-initialised from `seed` (last layer
 * scaled by 0.1), biases zero, Adam state zero. */
int fvm_closure_create(int n1, int n2, int n3, unsigned long long seed, fvm_closure** out);
int fvm_closure_destroy(fvm_closure* c);

/* Feature normalisation f = (prim - in_mean) / in_scale, output scales, and
 * loss weights per conserved variable; gamma of the gas. */
int fvm_closure_set_norm(fvm_closure* c, double gamma, const double in_mean[5], const double in_scale[5],
                         const double out_scale[5], const double loss_weight[5]);

/* Bound on the per-stage corrections: 0 = each face correction clipped to
 * +-beta*max(|v_a|+c)*|dU| only; 1 = that clip, then the flux-corrected
 * transport limiter (Zalesak): every face transfer is scaled so that the
 * corrected stage result stays inside the min/max of the plain stage result
 * over the cell and its six neighbours (no new extrema).  Set before
 * fvm_closure_attach (an attached step graph keeps the mode it was built with). */
int fvm_closure_set_limiter(fvm_closure* c, int fct);

/* layer in 1..3.  set_* resets that layer's Adam moments. */
int fvm_closure_set_weights(fvm_closure* c, int layer, const float* w_host, const float* b_host);
int fvm_closure_get_weights(fvm_closure* c, int layer, float* w_host, float* b_host);
/* Gradients of the last fvm_closure_backward. */
int fvm_closure_get_grads(fvm_closure* c, int layer, float* dw_host, float* db_host);

/* Copy a workspace buffer to (to_device = 0) or from (1) host memory; `bytes`
 * must equal the buffer size. */
int fvm_closure_buffer(fvm_closure* c, int which, void* host, long long bytes, int to_device);

/* Features of a dense float32 state [5][pos] on the device. */
int fvm_closure_features(fvm_closure* c, const float* u_dense_dev);
/* X0 -> A1 -> A2 -> Z3. */
int fvm_closure_forward(fvm_closure* c);
/* A-priori loss of Z3 against the target defect D (dense [5][pos], device):
 * E = dt * (-sum_a (dF(p) - dF(p - e_a)) / h_a) - D with dF = out_scale*Z3,
 * loss = sum w_q E^2 / N; then all weight and bias gradients. */
int fvm_closure_backward(fvm_closure* c, const float* defect_dense_dev, double dt, const double h[3]);
/* One Adam step on all layers (step counter advances). */
int fvm_closure_adam(fvm_closure* c, double lr, double beta1, double beta2, double eps);
/* features + forward + backward + adam. */
int fvm_closure_train_step(fvm_closure* c, const float* u_dense_dev, const float* defect_dense_dev, double dt,
                           const double h[3], double lr);
/* Device time per call (CUDA events on the closure's stream, one untimed
 * warm-up, `iters` back-to-back calls): the forward pass from the current
 * features, and the full training step (features, forward, loss, backward,
 * Adam -- the weights change). */
int fvm_closure_time_forward(fvm_closure* c, int iters, double* ms);
int fvm_closure_time_train(fvm_closure* c, const float* u_dense_dev, const float* defect_dense_dev, double dt,
                           const double h[3], double lr, int iters, double* ms);
/* Loss of the last backward (synchronises). */
int fvm_closure_loss(fvm_closure* c, double* out);

/* Apply the per-stage correction to dense states: uout += coef*dt*R where
 * R = -div(clip(out_scale*Z3)) with the clip bound taken from uin, cellwise
 * skipped where it would break positivity.  Uses the current Z3. */
int fvm_closure_correct_dense(fvm_closure* c, const float* uin_dense_dev, float* uout_dense_dev, double coef,
                              double dt, double beta, const double h[3], unsigned long long* n_switched);

/* Make every step of the solver handle h run the closure: Z3 from the step's
 * base state, then after each stage kernel the correction of the stage's
 * residual (clip factor beta).  Requires navier_stokes, float32, cartesian,
 * periodic on all faces, SSPRK3 or Euler, and h's grid equal to c's.  c may be
 * NULL to detach.  The closure must outlive the attachment. */
int fvm_closure_attach(fvm_handle* h, fvm_closure* c, double beta);
/* Number of cell-stage updates that kept the plain result since attach. */
int fvm_closure_switch_count(fvm_handle* h, unsigned long long* out);

/* f^3 box filter of h's float32 state into a dense coarse array (device). */
int fvm_filter_state(fvm_handle* h, int factor, float* coarse_dense_dev);
/* Interior of h's float32 state from / to a dense device array. */
int fvm_upload_dense(fvm_handle* h, const float* dense_dev);
int fvm_download_dense(fvm_handle* h, float* dense_dev);

#ifdef __cplusplus
}
#endif
#endif
