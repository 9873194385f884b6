// Flexible CG, the Chebyshev-Jacobi polynomial preconditioner (the fallback of the learned
// method) and the training pairs of the plain solver.  No counterpart in the reference, which
// solves with PETSc's CG and ILU (src/la/solve.cc:370).
#include <cuda_runtime.h>

#include "device_system.hpp"
#include "learned.hpp"

namespace mh {

namespace {

struct Plan {
    const int32_t *inst, *tile_begin, *tile_end, *inst_blk;
};

Plan plan32(const DevSystem &s) {
    const DevPlan &p = s.plan[1];
    return {p.blk_inst, p.tile_begin, p.tile_end, p.inst_blk};
}

template <int NV> struct Sums { double v[NV]; };

template <int NV> __device__ __forceinline__ Sums<NV> block_sum(Sums<NV> s) {
    __shared__ double sh[kWarpsPerBlock][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double v = s.v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) sh[warp][k] = v;
    }
    __syncthreads();
    Sums<NV> out;
#pragma unroll
    for (int k = 0; k < NV; ++k) out.v[k] = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarpsPerBlock; ++w)
#pragma unroll
            for (int k = 0; k < NV; ++k) out.v[k] += sh[w][k];
    __syncthreads();
    return out;
}

// Same contract as the Krylov kernels' block_finish (solver.cu): publish the block partial,
// the instance's last-arriving block gets the totals (thread 0).
template <int NV>
__device__ __forceinline__ bool block_finish(Sums<NV> s, double *partial, InstCtl *c, const Plan &plan, int inst,
                                             Sums<NV> &tot) {
    __shared__ bool am_last;
    Sums<NV> b = block_sum<NV>(s);
    const int pb = plan.inst_blk[inst], pe = plan.inst_blk[inst + 1];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partial[(int64_t)blockIdx.x * 4 + k] = b.v[k];
        __threadfence();
        am_last = (atomicAdd(&c->ticket, 1u) == (unsigned)(pe - pb) - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    Sums<NV> a;
#pragma unroll
    for (int k = 0; k < NV; ++k) a.v[k] = 0.0;
    for (int t = pb + threadIdx.x; t < pe; t += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) a.v[k] += __ldcg(&partial[(int64_t)t * 4 + k]);
    tot = block_sum<NV>(a);
    if (threadIdx.x == 0) c->ticket = 0u;
    return true;
}

__device__ __forceinline__ void finish_inst(InstCtl *c, int status, int32_t *n_done) {
    c->done = 1;
    c->status = status;
    atomicAdd(n_done, 1);
}

// a = (S^ h)[row] with float4 node states (FIRST: h = (r, 0, 0, 0) from a scalar vector)
template <bool FIRST>
__device__ __forceinline__ float4 aggregate(const SellView<float> &A, const float *__restrict__ r,
                                            const float4 *__restrict__ h, int64_t sl, int lane) {
    const int64_t off = A.slice_off[sl];
    const int w = (int)((A.slice_off[sl + 1] - off) / kSliceRows);
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = 0; j < w; ++j) {
        const int64_t slot = off + (int64_t)j * kSliceRows + lane;
        const float v = __ldcs(A.val + slot);
        const int32_t c = __ldcs(A.col + slot);
        if (FIRST) {
            acc.x += v * r[c];
        } else {
            const float4 hc = h[c];
            acc.x += v * hc.x;
            acc.y += v * hc.y;
            acc.z += v * hc.z;
            acc.w += v * hc.w;
        }
    }
    return acc;
}

// One layer of the network for the rows of the block's tiles (R = 1 tiles of 256 rows).
// FIRST: the input is the scalar residual; LAST: only channel 0 of the output is stored, as
// z, and the partial dot z.q_old of flexible CG is reduced (beta = z.q_old / (p.q)_old).
// ---- flexible CG ------------------------------------------------------------------------
// p = z - beta p; partial p.r -> rho (alpha = p.r / p.q is then formed by the SpMV kernel).
__global__ void __launch_bounds__(kBlockThreads)
    k_fcg_direction(const float *__restrict__ z, const float *__restrict__ r, float *__restrict__ p,
                    double *__restrict__ partial, InstCtl *__restrict__ ctl, Plan plan, int32_t *n_done) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (c->done) return;
    const double beta = c->beta;
    double pr = 0.0;
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        const int64_t row = (int64_t)tile * kBlockThreads + threadIdx.x;
        // beta = 0 starts a new direction sequence: p is not read (it may hold a broken one)
        const float pn = beta == 0.0 ? z[row] : (float)((double)z[row] - beta * (double)p[row]);
        p[row] = pn;
        pr += (double)pn * (double)r[row];
    }
    Sums<1> s = {{pr}};
    Sums<1> tot;
    if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
        c->rho = tot.v[0];
        if (!isfinite(tot.v[0])) finish_inst(c, -6, n_done);
    }
}

// x += alpha p; r -= alpha q; r.r and the stopping test.  Also keeps (p.q) for the next beta.
__global__ void __launch_bounds__(kBlockThreads)
    k_fcg_update(float *__restrict__ x, float *__restrict__ r, const float *__restrict__ p,
                 const float *__restrict__ q, double *__restrict__ partial, InstCtl *__restrict__ ctl, Plan plan,
                 int32_t *n_done) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (c->done) return;
    const double alpha = c->alpha;
    double rr = 0.0;
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        const int64_t row = (int64_t)tile * kBlockThreads + threadIdx.x;
        x[row] = (float)((double)x[row] + alpha * (double)p[row]);
        const float rn = (float)((double)r[row] - alpha * (double)q[row]);
        r[row] = rn;
        rr += (double)rn * (double)rn;
    }
    Sums<1> s = {{rr}};
    Sums<1> tot;
    if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
        c->aux[0] = c->rho / c->alpha;  // p.q of this iteration (alpha = p.r / p.q)
        c->aux[1] = 1.0;                // (p, q) hold a direction the next one is made conjugate to
        c->rr = tot.v[0];
        c->iter += 1;
        if (!isfinite(tot.v[0])) finish_inst(c, -6, n_done);
        else if (tot.v[0] <= c->tol2) finish_inst(c, 0, n_done);
        else if (c->iter >= c->max_it) finish_inst(c, 1, n_done);
    }
}

// ---- Chebyshev-Jacobi polynomial preconditioner z = P_d(S^) r on [lo, hi] ---------------
// step 0: d = r / theta, z = d;  step k: d = c1 d + c2 (r - S^ z_prev), z = z_prev + d.
// The last step also reduces z.q_old for the flexible-CG beta.
__global__ void __launch_bounds__(kBlockThreads)
    k_cheb_step(SellView<float> A, const float *__restrict__ r, const float *__restrict__ z_prev,
                float *__restrict__ z_next, float *__restrict__ d, double c1, double c2, int first,
                const float *__restrict__ q_old, double *__restrict__ partial, InstCtl *__restrict__ ctl, Plan plan,
                int32_t *n_done) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (c->done) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double zq = 0.0;
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        const int64_t sl = (int64_t)tile * kWarpsPerBlock + warp;
        const int64_t row = sl * kSliceRows + lane;
        float zn;
        if (first) {
            const float dn = (float)(c2 * (double)r[row]);
            d[row] = dn;
            zn = dn;
        } else {
            const float4 az = aggregate<true>(A, z_prev, nullptr, sl, lane);
            const double res = (double)r[row] - (double)az.x;
            const float dn = (float)(c1 * (double)d[row] + c2 * res);
            d[row] = dn;
            zn = z_prev[row] + dn;
        }
        z_next[row] = zn;
        if (q_old) zq += (double)zn * (double)q_old[row];
    }
    if (partial) {
        Sums<1> s = {{zq}};
        Sums<1> tot;
        if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0)
            c->beta = (c->aux[1] != 0.0 && c->aux[0] != 0.0) ? tot.v[0] / c->aux[0] : 0.0;
    }
}

// beta = z.q_old / (p.q)_old for flexible CG after a preconditioner that writes z only
__global__ void __launch_bounds__(kBlockThreads)
    k_fcg_beta(const float *__restrict__ z, const float *__restrict__ q_old, double *__restrict__ partial,
               InstCtl *__restrict__ ctl, Plan plan) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (c->done) return;
    double zq = 0.0;
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        const int64_t row = (int64_t)tile * kBlockThreads + threadIdx.x;
        zq += (double)z[row] * (double)q_old[row];
    }
    Sums<1> s = {{zq}};
    Sums<1> tot;
    if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0)
        c->beta = (c->aux[1] != 0.0 && c->aux[0] != 0.0) ? tot.v[0] / c->aux[0] : 0.0;
}

// Gershgorin bound max_i sum_j |S^_ij| (upper bound of the spectrum of S^)
__global__ void k_row_abs_max(SellView<float> A, int64_t n_rows, unsigned int *out) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.f;
    if (row < n_rows) {
        const int64_t sl = row / kSliceRows;
        const int lane = (int)(row % kSliceRows);
        const int64_t off = A.slice_off[sl];
        const int w = (int)((A.slice_off[sl + 1] - off) / kSliceRows);
        for (int j = 0; j < w; ++j) s += fabsf(A.val[off + (int64_t)j * kSliceRows + lane]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = fmaxf(s, __shfl_xor_sync(0xffffffffu, s, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(s));  // non-negative floats order as ints
}

// ---- training pairs of the plain solver --------------------------------------------
__global__ void k_pair_make(const double *__restrict__ xs, const double *__restrict__ x,
                            const double *__restrict__ r64, float *__restrict__ e, float *__restrict__ r, int64_t n,
                            double *acc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, er = 0.0;
    if (i < n) {
        const float ev = (float)(xs[i] - x[i]), rv = (float)r64[i];
        e[i] = ev;
        r[i] = rv;
        rr = (double)rv * (double)rv;
        er = (double)ev * (double)rv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        er += __shfl_xor_sync(0xffffffffu, er, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc, rr);
        atomicAdd(acc + 1, er);
    }
}

__global__ void k_pair_scale(float *__restrict__ e, float *__restrict__ r, float s, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        e[i] *= s;
        r[i] *= s;
    }
}

inline unsigned blocks_for(int64_t n, int th) { return (unsigned)((n + th - 1) / th); }

}  // namespace

// z = NN(r) on the FP32 inner vectors; with q_old the last layer reduces z.q_old -> beta.
cudaError_t launch_cheb_apply(const DevSystem &sys, const float *r, float *z0, float *z1, float *d, float *z_final,
                              const float *q_old, int degree, double lo, double hi, cudaStream_t s) {
    if (sys.rows_per_thread != 1) return cudaErrorInvalidValue;  // tiles of 256 rows
    const SellView<float> A = {sys.n_rows, sys.slice_off, sys.col, sys.val32};
    const unsigned g = (unsigned)sys.plan[1].n_blocks;
    const Plan p = plan32(sys);
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma;
    const float *zp = nullptr;
    for (int k = 0; k < degree; ++k) {
        double c1 = 0.0, c2 = 1.0 / theta;
        if (k > 0) {
            const double rho_new = 1.0 / (2.0 * sigma - rho);
            c1 = rho_new * rho;
            c2 = 2.0 * rho_new / delta;
            rho = rho_new;
        }
        const bool last = k == degree - 1;
        float *zn = last ? z_final : ((k % 2 == 0) ? z0 : z1);
        k_cheb_step<<<g, kBlockThreads, 0, s>>>(A, r, zp, zn, d, c1, c2, k == 0 ? 1 : 0, last ? q_old : nullptr,
                                                last && q_old ? sys.partial : nullptr, sys.ctl, p, sys.n_done);
        zp = zn;
    }
    return cudaGetLastError();
}

cudaError_t launch_fcg_beta(const DevSystem &sys, const float *z, const float *q_old, cudaStream_t s) {
    if (sys.rows_per_thread != 1) return cudaErrorInvalidValue;  // tiles of 256 rows
    k_fcg_beta<<<(unsigned)sys.plan[1].n_blocks, kBlockThreads, 0, s>>>(z, q_old, sys.partial, sys.ctl, plan32(sys));
    return cudaGetLastError();
}

cudaError_t launch_fcg_direction(const DevSystem &sys, const float *z, cudaStream_t s) {
    if (sys.rows_per_thread != 1) return cudaErrorInvalidValue;  // tiles of 256 rows
    k_fcg_direction<<<(unsigned)sys.plan[1].n_blocks, kBlockThreads, 0, s>>>(z, sys.r32, sys.p32, sys.partial, sys.ctl,
                                                                            plan32(sys), sys.n_done);
    return cudaGetLastError();
}

cudaError_t launch_fcg_update(const DevSystem &sys, cudaStream_t s) {
    if (sys.rows_per_thread != 1) return cudaErrorInvalidValue;  // tiles of 256 rows
    k_fcg_update<<<(unsigned)sys.plan[1].n_blocks, kBlockThreads, 0, s>>>(sys.x32, sys.r32, sys.p32, sys.q32,
                                                                         sys.partial, sys.ctl, plan32(sys), sys.n_done);
    return cudaGetLastError();
}

cudaError_t launch_spectrum_bound(const DevSystem &sys, unsigned int *out, cudaStream_t s) {
    const SellView<float> A = {sys.n_rows, sys.slice_off, sys.col, sys.val32};
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    k_row_abs_max<<<blocks_for(sys.n_rows, 256), 256, 0, s>>>(A, sys.n_rows, out);
    return cudaGetLastError();
}

// (r, e) of one training pair: e = x* - x, r = the solver's residual (FP32), with |r|^2 and
// e.r summed into acc
cudaError_t launch_pair_make(int64_t n, const double *xs, const double *x, const double *r64, float *e, float *r,
                             double *acc, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(acc, 0, 2 * sizeof(double), s);
    if (err != cudaSuccess) return err;
    k_pair_make<<<blocks_for(n, 256), 256, 0, s>>>(xs, x, r64, e, r, n, acc);
    return cudaGetLastError();
}

cudaError_t launch_pair_scale(int64_t n, float *e, float *r, float scale, cudaStream_t s) {
    k_pair_scale<<<blocks_for(n, 256), 256, 0, s>>>(e, r, scale, n);
    return cudaGetLastError();
}

}  // namespace mh
