// Learned smoother network (smoother_nn.cu): sizes, parameter layout and launchers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device_system.hpp"

namespace mh {

constexpr int kSnW = 32;  // width
constexpr int kSnF = 8;   // row features
constexpr int kSnL = 3;   // message-passing layers
constexpr int kSnPerLayer = kSnW * 2 * kSnW + kSnW;  // W_l [32][64], b_l [32]
constexpr int kSnOffW0 = 0, kSnOffB0 = kSnW * kSnF, kSnOffLayer = kSnOffB0 + kSnW;
constexpr int kSnOffWout = kSnOffLayer + kSnL * kSnPerLayer, kSnOffBout = kSnOffWout + kSnW;
constexpr int kSnParams = kSnOffBout + 1;  // 6561
constexpr int kSnWgradBlocks = 296;        // row blocks of the weight-gradient partials

// Activations over the solver rows, [n][32] each (u: pre-activations, kept for training)
struct SnActs {
    float *h[kSnL + 1] = {};
    float *a[kSnL] = {};
    float *u[kSnL] = {};
    float *u0 = nullptr, *z = nullptr;
};

struct SnScratch {
    float *dz = nullptr;                       // [n]
    float *dh = nullptr, *du = nullptr, *da = nullptr;  // [n][32]
    float *part = nullptr;                     // [kSnWgradBlocks][2080]
};

// x [n][8] row features of the solver's FP32 matrix
cudaError_t sn_features(const DevSystem &sys, float *x, cudaStream_t s);
// smoother weights w [n] (1 on padding rows); keep: store every activation for sn_backward
// (else only h[0], h[1] and a[0] are used)
cudaError_t sn_forward(const DevSystem &sys, const float *params, const float *x, SnActs &act, float *w, bool keep,
                       cudaStream_t s);
// grad [kSnParams] of a loss whose derivative with respect to w is dw [n]
cudaError_t sn_backward(const DevSystem &sys, const float *params, const float *x, SnActs &act, const float *dw,
                        float *grad, SnScratch &sc, cudaStream_t s);
cudaError_t sn_adam(float *params, float *m, float *v, const float *grad, int step, float lr, cudaStream_t s);
// pieces of the smoother gradient
cudaError_t sn_spmv(const DevSystem &sys, const float *w, const float *v, float *y, cudaStream_t s);
cudaError_t sn_axpy(int64_t n, const float *a, float alpha, const float *b, float *out, cudaStream_t s);
cudaError_t sn_dot(int64_t n, const float *x, const float *y, double *part, double *out, cudaStream_t s);
cudaError_t sn_grad_w(const DevSystem &sys, float a0, float a1, const float *g, const float *h, const float *r,
                      const float *r2, const float *swr, const float *swr2, const float *swg, const float *swh,
                      const int32_t *agg, float scale, float *dw, cudaStream_t s);

}  // namespace mh
