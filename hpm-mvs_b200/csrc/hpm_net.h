/*
 * Launchers of the proposal network's tensor-core kernels (hpm_net.cu) for
 * the prior-net form (hpm_priornet.cu).  All asynchronous on `s`.
 */
#pragma once

#include <cuda_runtime.h>

namespace hpm {

/* 3x3 convolution of NHWC BF16 activations (epilogue 0: ReLU to BF16, 1:
 * bias to FP32, 2: ReLU gradient to BF16); err is set when a wait ran out. */
cudaError_t net_conv3x3(const void *x, int h, int w, int cin, const void *wpk, const float *bias, int cout, int epi,
                        const void *aux, void *y, int *err, bool use_tma, cudaStream_t s);
cudaError_t net_pack_weights(const float *wt, int cout, int cin, int mode, void *out, cudaStream_t s);
cudaError_t net_conv_wgrad(const void *x, const void *dy, int h, int w, int cin, int cout, float *dw, int *err,
                           int ctas, cudaStream_t s);
cudaError_t net_bias_grad(const void *dy, int is_f32, long long n, int c, float *db, cudaStream_t s);

}  // namespace hpm
