// Learned preconditioner (K7), flexible CG and Chebyshev-Jacobi: declarations shared by
// learned.cu and the host runtime.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device_system.hpp"

namespace mh {

constexpr int kNnK = 4;                // node state channels
constexpr int kNnH = 32;               // MLP width
constexpr int kNnLayers = 3;
constexpr int kNnPerLayer = kNnH * 2 * kNnK + kNnH + kNnK * kNnH + kNnK;  // 420: W1, b1, W2, b2
constexpr int kNnParams = kNnLayers * kNnPerLayer;
constexpr int kNnPackedPerLayer = 128 + 64;  // bf16 pairs of W1 (32x8) and W2 (4x32)

// Device view of one layer for the tensor-core inference kernel.
struct NnLayerView {
    const uint32_t *w1b, *w2b;  // bf16x2 words
    const float *b1, *b2;
};

// Activations kept by a training pass (rows of the padded solver space).
struct NnTrainBuffers {
    float4 *h[kNnLayers + 1];
    float4 *a[kNnLayers];
    float4 *g[2];
    float4 *ga;
    float *z;
};

NnLayerView nn_layer_view(const float *w, const uint32_t *wb, int l);
cudaError_t launch_nn_pack(const float *w, uint32_t *wb, cudaStream_t s);
cudaError_t launch_nn_apply(const DevSystem &sys, const float *w, const uint32_t *wb, const float *r, float4 *h0,
                            float4 *h1, float *z, const float *q_old, cudaStream_t s);
cudaError_t launch_cheb_apply(const DevSystem &sys, const float *r, float *z0, float *z1, float *d, float *z_final,
                              const float *q_old, int degree, double lo, double hi, cudaStream_t s);
// beta of flexible CG from z and the previous q (for preconditioners that only write z)
cudaError_t launch_fcg_beta(const DevSystem &sys, const float *z, const float *q_old, cudaStream_t s);
cudaError_t launch_fcg_direction(const DevSystem &sys, const float *z, cudaStream_t s);
cudaError_t launch_fcg_update(const DevSystem &sys, cudaStream_t s);
cudaError_t launch_spectrum_bound(const DevSystem &sys, unsigned int *out, cudaStream_t s);
cudaError_t launch_nn_train_pair(const DevSystem &sys, const float *w, const float *r, const float *e, double er,
                                 NnTrainBuffers &b, float *grad, double *loss, cudaStream_t s);
cudaError_t launch_nn_adam(float *w, float *m, float *v, const float *grad, int step, float lr, float scale,
                           int train_bias, cudaStream_t s);
cudaError_t launch_pair_make(int64_t n, const double *xs, const double *x, const double *r64, float *e, float *r,
                             double *acc, cudaStream_t s);
cudaError_t launch_pair_scale(int64_t n, float *e, float *r, float scale, cudaStream_t s);

}  // namespace mh
