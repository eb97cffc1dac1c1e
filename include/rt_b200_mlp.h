/* rt_b200_mlp.h -- the coordinate MLP of the learned warm start.
 *
 * No reference counterpart.  A coordinate MLP predicts a domain's mean height
 * surface from per-vertex features; its prediction is projected onto a valid
 * height function (rt_b200_project.h) and turned into the start tiling of a
 * plain chain.  Architecture: IN = 8 input features -> 128 -> 128 -> 128 -> 1,
 * GELU (tanh form) after each hidden layer.  The two 128 x 128 layers run on
 * the tensor cores (tcgen05.mma, accumulators in tensor memory) in BF16 with
 * FP32 accumulation (forward, and both GEMMs of the backward pass); the
 * 8 -> 128 and 128 -> 1 layers and Adam run in FP32.
 * Master parameters are FP32; BF16 copies of the 128 x 128 weights are made
 * after every update.  Loss: mean squared error.
 *
 * Parameter vector layout (RT_MLP_PARAMS floats):
 *   W0[128][8], b0[128], W1[128][128], b1[128], W2[128][128], b2[128], W3[128], b3[1]
 * (W[out][in]).
 */
#ifndef RT_B200_MLP_H
#define RT_B200_MLP_H

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RT_MLP_IN 8
#define RT_MLP_WIDTH 128
#define RT_MLP_PARAMS (128 * 8 + 128 + 128 * 128 + 128 + 128 * 128 + 128 + 128 + 1)

typedef struct rt_mlp rt_mlp;

rt_status rt_mlp_create(int32_t device, uint64_t seed, rt_mlp** out);
rt_status rt_mlp_destroy(rt_mlp* m);
/* Copies the FP32 master parameters to / from the host (RT_MLP_PARAMS floats). */
rt_status rt_mlp_get_params(rt_mlp* m, float* params);
rt_status rt_mlp_set_params(rt_mlp* m, const float* params);
/* Forward pass of n rows of RT_MLP_IN features (host, row-major) into y (n floats). */
rt_status rt_mlp_predict(rt_mlp* m, const float* x, int64_t n, float* y);
/* Loss and gradient (RT_MLP_PARAMS floats, FP32) of one batch; parameters unchanged. */
rt_status rt_mlp_loss_grad(rt_mlp* m, const float* x, const float* target, int64_t n, float* loss, float* grad);
/* Uploads a training set (n rows) that rt_mlp_train samples batches from. */
rt_status rt_mlp_set_data(rt_mlp* m, const float* x, const float* target, int64_t n);
/* `steps` Adam steps (lr, beta1 0.9, beta2 0.999, eps 1e-8) on batches of
 * `batch` rows drawn uniformly with replacement from the training set
 * (counter-based draws keyed by `seed`); *loss gets the mean loss of the last
 * step. */
rt_status rt_mlp_train(rt_mlp* m, int64_t steps, int32_t batch, float lr, uint64_t seed, float* loss);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_MLP_H */
