/*
 * tslb_closure.h -- learned eddy-viscosity closure for coarse TSLB grids.
 *
 * The reference has no counterpart: its coarse-grid runs (the turbulent jet
 * of boundary_cds_3D_module.f90:862-1119 driven by recursive_2c_TSLB3D.f90)
 * use the plain relaxation time.  This closure corrects the local relaxation
 * time of a colour-mode lattice with a small network evaluated on the GPU
 * every step (or every `interval` steps):
 *
 *   tau_x = tau(phi_x) + dtau_x,   dtau_x = dtau_min + (dtau_max - dtau_min) sigmoid(o_x),
 *   o = w3 . relu(W2 relu(W1 xn + b1) + b2) + b3,   xn = (f - mu) / sd,
 *
 * with the 10 features f of node x (all from the lattice's own moments):
 *   f0..f5  s * Pi^neq (xx, xy, xz, yy, yz, zz),  s = tau(phi)/(tau(phi) + dtau_prev)
 *           rescales the stored non-equilibrium stress to the plain tau,
 *   f6      phi,
 *   f7      |grad phi| by central differences (periodic faces wrap, other
 *           faces repeat the boundary node),
 *   f8      |u|,
 *   f9      s * |Pi^neq|_F = s * sqrt(Pxx^2 + Pyy^2 + Pzz^2 + 2 (Pxy^2 + Pxz^2 + Pyz^2)).
 *
 * The dense layers run on the tensor cores (tcgen05, BF16 operands, FP32
 * accumulation in tensor memory); W1, W2, w3 are rounded to BF16, biases
 * stay FP32.  Stability clamp: a node whose features or output are not
 * finite keeps the plain tau (dtau = 0); dtau is clamped to [dtau_min,
 * dtau_max].  dtau_min is 0 unless set (a negative dtau_min lets the
 * network lower the viscosity; attaching checks tau + dtau_min > 1/2).
 *
 * Training (tslb_closure_train) runs forward and backward passes on the
 * tensor cores and updates FP32 master weights with Adam.  The loss of a
 * sample (features f, target t, weight a) is a (y - t)^2 averaged over the
 * batch, y the network's dtau.  Samples come from box-filtered fine-grid
 * states (tslb_closure_dataset_add_fine): t = 3 nu_t is the eddy viscosity
 * that best fits the subgrid stress of the factor-2 box filter,
 *   nu_t = -(tau^sgs_dev : S) / (2 S : S),  a = S : S,
 * tau^sgs = mean(u u) - mean(u) mean(u) over each 2x2x2 block and S the
 * strain rate of the filtered velocity on the coarse grid.
 *
 * Parameter vector (FP32, TSLB_CLOSURE_NPARAM values):
 *   W1[64][16] at TSLB_CLOSURE_OFF_W1 (row = hidden unit, column = feature;
 *   columns 10..15 are padding and stay 0), b1[64], W2[64][64] (row =
 *   output unit), b2[64], w3[64], b3.
 *
 * Every function returns TSLB_OK (0) or a TSLB_ERR_* code and never aborts;
 * tslb_closure_last_error() gives the message.  Host arrays are borrowed for
 * the call.  Feature arrays are row-major n x 10.
 */
#ifndef TSLB_CLOSURE_H
#define TSLB_CLOSURE_H

#include "tslb.h"

#ifdef __cplusplus
extern "C" {
#endif

#define TSLB_CLOSURE_NFEAT   10
#define TSLB_CLOSURE_HIDDEN  64
#define TSLB_CLOSURE_OFF_W1  0
#define TSLB_CLOSURE_OFF_B1  1024
#define TSLB_CLOSURE_OFF_W2  1088
#define TSLB_CLOSURE_OFF_B2  5184
#define TSLB_CLOSURE_OFF_W3  5248
#define TSLB_CLOSURE_OFF_B3  5312
#define TSLB_CLOSURE_NPARAM  5313

typedef struct tslb_closure tslb_closure;

/* A closure on the current device with all parameters 0, mu = 0, sd = 1,
 * dtau_max = 0.01. */
int  tslb_closure_create(tslb_closure** out);
void tslb_closure_destroy(tslb_closure* c);

/* Parameters (FP32 master copy), feature normalisation and output bound.
 * Any pointer of set_params may be NULL to keep that part. */
int  tslb_closure_set_params(tslb_closure* c, const float* params, const float* mu, const float* sd, float dtau_max);
int  tslb_closure_get_params(tslb_closure* c, float* params, float* mu, float* sd, float* dtau_max);
/* Lower bound of the output, dtau_min <= 0 (0 after create). */
int  tslb_closure_set_dtau_min(tslb_closure* c, float dtau_min);
float tslb_closure_dtau_min(const tslb_closure* c);

/* dtau of n feature rows (host arrays). */
int  tslb_closure_forward(tslb_closure* c, const float* features, long long n, float* dtau);

/* Gradient of the mean loss over n samples (one batch) with respect to the
 * parameter vector, and the loss itself, without updating anything. */
int  tslb_closure_gradient(tslb_closure* c, const float* features, const float* target, const float* weight,
                           long long n, float* grad, double* loss);

/* ---- training set, kept on the device ---- */
int  tslb_closure_dataset_clear(tslb_closure* c);
int  tslb_closure_dataset_add(tslb_closure* c, const float* features, const float* target, const float* weight,
                              long long n);
/* Samples of a fine colour-mode lattice (FP32 storage, even sizes) filtered
 * onto the grid of half its size: every keep_every-th coarse node of the
 * coarse planes z_lo <= z < z_hi (z_hi <= 0: to the last plane), starting
 * at an offset that cycles with each call; Pi^neq is multiplied by pi_scale
 * to express it at the coarse grid's plain tau (2 tau_coarse / tau_fine for
 * acoustic scaling).  *added (may be NULL) receives the number of samples
 * appended. */
int  tslb_closure_dataset_add_fine(tslb_closure* c, tslb_ctx* fine, float pi_scale, int keep_every,
                                   int z_lo, int z_hi, long long* added);
long long tslb_closure_dataset_size(tslb_closure* c);
int  tslb_closure_dataset_download(tslb_closure* c, float* features, float* target, float* weight);
/* mu, sd of the features over the training set; weights rescaled to mean 1. */
int  tslb_closure_normalize(tslb_closure* c);

/* Adam on the training set: `steps` steps of `batch` samples (a multiple of
 * 128) drawn with a counter-based hash of (seed, step, slot); the learning
 * rate decays from lr to lr/10 on a cosine.  loss_history (may be NULL)
 * receives the batch loss of each step. */
int  tslb_closure_train(tslb_closure* c, int steps, int batch, float lr, unsigned long long seed,
                        float* loss_history);

/* Raw features (n x 10) of every node of a colour-mode FP32 lattice. */
int  tslb_closure_features(tslb_closure* c, tslb_ctx* lattice, float* features);

/* Attach (c != NULL) or detach (c == NULL) the closure: before every
 * `interval`-th step the lattice refreshes its per-node tau correction from
 * the closure on its own stream: dtau = static field (tslb_set_tau_correction,
 * if set) + the network's output; the features' s uses the previous total.
 * The closure must outlive the attachment; do not train or change an
 * attached closure while the lattice's stream has work queued. */
int  tslb_attach_closure(tslb_ctx* lattice, tslb_closure* c, int interval);

/* Message of the last failed call on c (or, when c is NULL, of the calling
 * thread's last failed tslb_closure_create).  Never NULL. */
const char* tslb_closure_last_error(tslb_closure* c);

#ifdef __cplusplus
}
#endif

#endif /* TSLB_CLOSURE_H */
