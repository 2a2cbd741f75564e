/* gpe_cnn.h -- C-ABI of the learned coarse-grid correction (no reference
 * counterpart: the reference has no learned component).
 *
 * The network: 4 conv3d layers with 3x3x3 kernels and periodic padding,
 * channels 2 -> 16 -> 16 -> 16 -> 2, GELU after the first three, BF16
 * weights and activations with FP32 accumulation on the tcgen05 tensor
 * cores.  Input: Re/Im psi of a coarse grid; output: a correction
 * delta = out_scale * net(psi) added to psi after each coarse time step.
 *
 * Weights are exchanged as FP32 arrays w[4][27][16 co][16 ci] (tap index
 * (dz+1)*9 + (dy+1)*3 + (dx+1), applied as out(p) = sum w * in(p + (dx,dy,dz)))
 * and b[4][16]; entries outside a layer's real channels (ci >= 2 of layer 0,
 * co >= 2 of layer 3) are ignored and kept zero.
 *
 * All work is stream-ordered on the given context's stream; every call
 * returns after that stream has finished it, except gpe_cnn_attach's
 * per-step corrections, which are enqueued with the context's steps.
 * Grid limits: periodic grids (bcs 1), complex64 contexts, nx a multiple of
 * 16 and at most 128. */
#ifndef GPE_CNN_H
#define GPE_CNN_H

#include <stdint.h>

#include "gpe_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpe_cnn gpe_cnn;

typedef struct gpe_cnn_params {
  int32_t struct_size;   /* sizeof(gpe_cnn_params) */
  int32_t nx, ny, nz;    /* coarse grid */
  int32_t device;
  int32_t train;         /* 1: allocate training buffers */
  float out_scale;       /* delta = out_scale * last layer output (default 0.01) */
  int32_t preserve_norm; /* 1: after each attached correction, psi is rescaled
                            to the norm of the step it corrects (the
                            correction then moves no mass) */
} gpe_cnn_params;

#define GPE_CNN_LAYERS 4
#define GPE_CNN_TAPS 27
#define GPE_CNN_CH 16
#define GPE_CNN_WEIGHTS (GPE_CNN_LAYERS * GPE_CNN_TAPS * GPE_CNN_CH * GPE_CNN_CH)
#define GPE_CNN_BIASES (GPE_CNN_LAYERS * GPE_CNN_CH)

void gpe_cnn_default_params(gpe_cnn_params* p, int32_t nx, int32_t ny, int32_t nz);
int gpe_cnn_create(const gpe_cnn_params* p, gpe_cnn** out);
void gpe_cnn_destroy(gpe_cnn* cnn);
const char* gpe_cnn_last_error(const gpe_cnn* cnn);

/* Host FP32 weights in / out (layouts above). */
int gpe_cnn_set_weights(gpe_cnn* cnn, const float* w, const float* b);
int gpe_cnn_get_weights(const gpe_cnn* cnn, float* w, float* b);

/* psi += delta(psi) on the context's resident field (inference path). */
int gpe_cnn_apply(gpe_cnn* cnn, gpe_ctx* ctx);
/* Apply the correction after every later step of ctx (gpe_gpu_solver /
 * gpe_gpu_advance); cnn == NULL detaches.  The per-step norms those calls
 * report are of the state before the correction. */
int gpe_cnn_attach(gpe_cnn* cnn, gpe_ctx* ctx);

/* Training-path forward: delta of the context's psi into delta_dev (device,
 * dense float [nz][ny][nx][2]); psi is not changed. */
int gpe_cnn_delta(gpe_cnn* cnn, gpe_ctx* ctx, float* delta_dev);
/* Loss of one pair and its gradients: u = the context's psi (a coarse step's
 * result), target_dev = dense complex interior array (elem_bytes 8 or 16);
 * loss = mean over sites of |u + delta(u) - target|^2.  dw, db: host arrays
 * of the weight layout (may be NULL). */
int gpe_cnn_grad(gpe_cnn* cnn, gpe_ctx* ctx, const void* target_dev, int32_t elem_bytes,
                 double* loss, float* dw, float* db);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the same loss. */
int gpe_cnn_train_step(gpe_cnn* cnn, gpe_ctx* ctx, const void* target_dev,
                       int32_t elem_bytes, float lr, double* loss);
int gpe_cnn_adam_reset(gpe_cnn* cnn);

/* 2:1 restriction (2x2x2 average) of a fine context's psi into a dense
 * complex device array of the half-size grid (elem_bytes 8 or 16). */
int gpe_cnn_restrict(gpe_ctx* fine, void* coarse_dev, int32_t elem_bytes);

int64_t gpe_cnn_launch_count(const gpe_cnn* cnn);

#ifdef __cplusplus
}
#endif

#endif /* GPE_CNN_H */
