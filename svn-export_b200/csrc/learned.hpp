// Flexible CG, Chebyshev-Jacobi and the training pairs of the plain solver (learned.cu):
// declarations shared with the host runtime.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device_system.hpp"

namespace mh {

cudaError_t launch_cheb_apply(const DevSystem &sys, const float *r, float *z0, float *z1, float *d, float *z_final,
                              const float *q_old, int degree, double lo, double hi, cudaStream_t s);
// beta of flexible CG from z and the previous q (for preconditioners that only write z)
cudaError_t launch_fcg_beta(const DevSystem &sys, const float *z, const float *q_old, cudaStream_t s);
cudaError_t launch_fcg_direction(const DevSystem &sys, const float *z, cudaStream_t s);
cudaError_t launch_fcg_update(const DevSystem &sys, cudaStream_t s);
cudaError_t launch_spectrum_bound(const DevSystem &sys, unsigned int *out, cudaStream_t s);
cudaError_t launch_pair_make(int64_t n, const double *xs, const double *x, const double *r64, float *e, float *r,
                             double *acc, cudaStream_t s);
cudaError_t launch_pair_scale(int64_t n, float *e, float *r, float scale, cudaStream_t s);

}  // namespace mh
