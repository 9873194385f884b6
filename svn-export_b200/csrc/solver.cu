// K2/K3/K5: Krylov kernels on the SELL-C-sigma edge system.
//
// Replaces KSPSolve on schur2 (src/la/solve.cc:447-460: PETSc CG).  The system is solved in
// the symmetrically diagonal-scaled form  S^ = D^-1/2 S D^-1/2  (Jacobi-preconditioned CG
// written as plain CG on S^), so no preconditioner vector is streamed.  One CG iteration is
// two kernels:
//   spmv:   q = S^ p, with partial sums p.q, r.q, q.q; the instance's last block computes
//           alpha = rho/(p.q) and beta from rho_new = rho - 2 alpha r.q + alpha^2 q.q;
//   update: x += alpha p, r -= alpha q, p = r + beta p, partial r.r; the last block stores the
//           exact rho for the next alpha and applies the stopping test.
// Reductions are deterministic: each tile writes a partial, the last-arriving block of an
// instance (atomic ticket, no spin-waits) sums that instance's partials in a fixed order.
// Tiles never straddle instances, so a batch of independent systems shares every launch and
// each keeps its own alpha/beta/convergence (per-instance masks).
#include <cuda_runtime.h>

#include "device_system.hpp"

namespace mh {

namespace {

template <int NV> struct Sums { double v[NV]; };

// Block-wide sum of NV doubles; result valid in thread 0.
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
    if (threadIdx.x == 0) {
        for (int w = 0; w < kWarpsPerBlock; ++w)
#pragma unroll
            for (int k = 0; k < NV; ++k) out.v[k] += sh[w][k];
    }
    __syncthreads();
    return out;
}

// Writes this tile's partial sums and returns true in every thread of the block that
// arrived last for its instance; that block then holds the instance totals in `tot`
// (thread 0 only).
template <int NV>
__device__ __forceinline__ bool tile_finish(Sums<NV> s, double *partial, InstCtl *c, int tile, Sums<NV> &tot) {
    __shared__ bool am_last;
    Sums<NV> b = block_sum<NV>(s);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partial[(int64_t)tile * 4 + k] = b.v[k];
        __threadfence();
        const unsigned n_tiles = (unsigned)(c->tile_end - c->tile_begin);
        const unsigned t = atomicAdd(&c->ticket, 1u);
        am_last = (t == n_tiles - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    Sums<NV> a;
#pragma unroll
    for (int k = 0; k < NV; ++k) a.v[k] = 0.0;
    for (int t = c->tile_begin + threadIdx.x; t < c->tile_end; t += blockDim.x)
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

template <typename T> __device__ __forceinline__ T ldg_stream(const T *p) { return __ldcs(p); }

// q = S^ p and the three dot products.
template <typename T, int R>
__global__ void __launch_bounds__(kBlockThreads) k_cg_spmv(SellView<T> A, const T *__restrict__ p, T *__restrict__ q,
                                                           const T *__restrict__ r, double *__restrict__ partial,
                                                           InstCtl *__restrict__ ctl, const int32_t *__restrict__ tile_inst,
                                                           int32_t *n_done) {
    const int tile = blockIdx.x;
    InstCtl *c = ctl + tile_inst[tile];
    if (c->done) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sums<3> s = {{0.0, 0.0, 0.0}};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t sl = ((int64_t)tile * kWarpsPerBlock + warp) * R + k;
        const int64_t off = A.slice_off[sl];
        const int w = (int)((A.slice_off[sl + 1] - off) / kSliceRows);
        const int64_t row = sl * kSliceRows + lane;
        double y = 0.0;
        const T *vv = A.val + off + lane;
        const int32_t *cc = A.col + off + lane;
        for (int j = 0; j < w; ++j) y += (double)ldg_stream(vv + j * kSliceRows) * (double)p[ldg_stream(cc + j * kSliceRows)];
        q[row] = (T)y;
        const double pr = (double)p[row], rr = (double)r[row];
        s.v[0] += pr * y;
        s.v[1] += rr * y;
        s.v[2] += y * y;
    }
    Sums<3> tot;
    if (tile_finish<3>(s, partial, c, tile, tot) && threadIdx.x == 0) {
        const double pq = tot.v[0], rq = tot.v[1], qq = tot.v[2];
        const double rho = c->rho;
        if (rho == 0.0) {
            c->alpha = 0.0;
            c->beta = 0.0;
            finish_inst(c, 0, n_done);
        } else if (!(pq > 0.0) || !isfinite(pq)) {
            c->alpha = 0.0;
            c->beta = 0.0;
            finish_inst(c, isfinite(pq) ? -8 : -6, n_done);
        } else {
            const double alpha = rho / pq;
            double rho_new = rho - 2.0 * alpha * rq + alpha * alpha * qq;
            if (rho_new < 0.0) rho_new = 0.0;
            c->alpha = alpha;
            c->beta = rho_new / rho;
        }
    }
}

// x += alpha p; r -= alpha q; p = r + beta p; r.r
template <typename T, int R>
__global__ void __launch_bounds__(kBlockThreads) k_cg_update(T *__restrict__ x, T *__restrict__ r, T *__restrict__ p,
                                                             const T *__restrict__ q, double *__restrict__ partial,
                                                             InstCtl *__restrict__ ctl,
                                                             const int32_t *__restrict__ tile_inst, int32_t *n_done) {
    const int tile = blockIdx.x;
    InstCtl *c = ctl + tile_inst[tile];
    if (c->done) return;
    const double alpha = c->alpha, beta = c->beta;
    Sums<1> s = {{0.0}};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t row = ((int64_t)tile * R + k) * kBlockThreads + threadIdx.x;
        const double pr = (double)p[row];
        const double xr = (double)x[row] + alpha * pr;
        const double rr = (double)r[row] - alpha * (double)ldg_stream(q + row);
        x[row] = (T)xr;
        r[row] = (T)rr;
        p[row] = (T)(rr + beta * pr);
        const double rs = (double)(T)rr;
        s.v[0] += rs * rs;
    }
    Sums<1> tot;
    if (tile_finish<1>(s, partial, c, tile, tot) && threadIdx.x == 0) {
        const double rr = tot.v[0];
        c->rho = rr;
        c->rr = rr;
        c->iter += 1;
        if (!isfinite(rr)) finish_inst(c, -6, n_done);
        else if (rr <= c->tol2) finish_inst(c, 0, n_done);
        else if (c->iter >= c->max_it) finish_inst(c, 1, n_done);
    }
}

// r = b - S^ x; p = r; start a CG run.  tol2 = max(rtol2 * (use_b ? b.b : r.r), atol2).
// With use_active, instances whose flag inst_sums[kSumStride*i + kSumActive] is 0 are marked done at once.
template <typename T, int R>
__global__ void __launch_bounds__(kBlockThreads) k_cg_init(SellView<T> A, const T *__restrict__ b, const T *__restrict__ x,
                                                           T *__restrict__ r, T *__restrict__ p,
                                                           double *__restrict__ partial, InstCtl *__restrict__ ctl,
                                                           const int32_t *__restrict__ tile_inst, int32_t *n_done,
                                                           int use_b, double rtol2, double atol2, int max_it,
                                                           const double *__restrict__ inst_sums, int use_active) {
    const int tile = blockIdx.x;
    const int inst = tile_inst[tile];
    InstCtl *c = ctl + inst;
    const bool active = !use_active || inst_sums[kSumStride * inst + kSumActive] != 0.0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sums<2> s = {{0.0, 0.0}};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t sl = ((int64_t)tile * kWarpsPerBlock + warp) * R + k;
        const int64_t off = A.slice_off[sl];
        const int w = (int)((A.slice_off[sl + 1] - off) / kSliceRows);
        const int64_t row = sl * kSliceRows + lane;
        double y = 0.0;
        for (int j = 0; j < w; ++j) {
            const int64_t slot = off + (int64_t)j * kSliceRows + lane;
            y += (double)A.val[slot] * (double)x[A.col[slot]];
        }
        const double bb = (double)b[row];
        const double rr = bb - y;
        r[row] = (T)rr;
        p[row] = (T)rr;
        s.v[0] += rr * rr;
        s.v[1] += bb * bb;
    }
    Sums<2> tot;
    if (tile_finish<2>(s, partial, c, tile, tot) && threadIdx.x == 0) {
        const double rr = tot.v[0], bb = tot.v[1];
        c->rho = rr;
        c->rr = rr;
        c->rr0 = rr;
        c->alpha = 0.0;
        c->beta = 0.0;
        c->iter = 0;
        c->max_it = max_it;
        c->status = 0;
        c->done = 0;
        const double ref = use_b ? bb : rr;
        c->tol2 = fmax(rtol2 * ref, atol2);
        if (!active) finish_inst(c, 0, n_done);
        else if (!isfinite(rr)) finish_inst(c, -6, n_done);
        else if (rr <= c->tol2) finish_inst(c, 0, n_done);
    }
}

// FP64 true residual r = bh - S^ x, with per-instance sums
//   {r.r, sum d r^2, sum d bh^2, bh.bh}
// (d = diag S: the middle two are the squared norms of the unscaled residual and rhs, the
// outer two those of the Jacobi-scaled ones).
template <int R>
__global__ void __launch_bounds__(kBlockThreads) k_residual64(SellView<double> A, const double *__restrict__ bh,
                                                              const double *__restrict__ x, const double *__restrict__ dsq,
                                                              double *__restrict__ r, double *__restrict__ partial,
                                                              InstCtl *__restrict__ ctl,
                                                              const int32_t *__restrict__ tile_inst,
                                                              double *__restrict__ inst_sums) {
    const int tile = blockIdx.x;
    const int inst = tile_inst[tile];
    InstCtl *c = ctl + inst;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Sums<4> s = {{0.0, 0.0, 0.0, 0.0}};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t sl = ((int64_t)tile * kWarpsPerBlock + warp) * R + k;
        const int64_t off = A.slice_off[sl];
        const int w = (int)((A.slice_off[sl + 1] - off) / kSliceRows);
        const int64_t row = sl * kSliceRows + lane;
        double y = 0.0;
        for (int j = 0; j < w; ++j) {
            const int64_t slot = off + (int64_t)j * kSliceRows + lane;
            y += A.val[slot] * x[A.col[slot]];
        }
        const double b = bh[row];
        const double rr = b - y;
        r[row] = rr;
        const double d = dsq[row] * dsq[row];
        s.v[0] += rr * rr;
        s.v[1] += d * rr * rr;
        s.v[2] += d * b * b;
        s.v[3] += b * b;
    }
    Sums<4> tot;
    if (tile_finish<4>(s, partial, c, tile, tot) && threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) inst_sums[kSumStride * inst + k] = tot.v[k];
    }
}

// Start an FP32 inner solve of S^ d = r / |r| for every instance whose outer residual is
// above its target (inst_sums[kSumStride*i + kSumActive] = 1 marks an active instance).
template <int R>
__global__ void __launch_bounds__(kBlockThreads) k_ir_start(const double *__restrict__ r64, float *__restrict__ x32,
                                                            float *__restrict__ r32, float *__restrict__ p32,
                                                            double *__restrict__ partial, InstCtl *__restrict__ ctl,
                                                            const int32_t *__restrict__ tile_inst,
                                                            const double *__restrict__ inst_sums, int32_t *n_done,
                                                            double rtol2, int max_it) {
    const int tile = blockIdx.x;
    const int inst = tile_inst[tile];
    InstCtl *c = ctl + inst;
    const bool active = inst_sums[kSumStride * inst + kSumActive] != 0.0;
    const double nrm = sqrt(inst_sums[kSumStride * inst + 0]);
    const double inv = (active && nrm > 0.0) ? 1.0 / nrm : 0.0;
    Sums<1> s = {{0.0}};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t row = ((int64_t)tile * R + k) * kBlockThreads + threadIdx.x;
        const float v = (float)(r64[row] * inv);
        x32[row] = 0.0f;
        r32[row] = v;
        p32[row] = v;
        s.v[0] += (double)v * (double)v;
    }
    Sums<1> tot;
    if (tile_finish<1>(s, partial, c, tile, tot) && threadIdx.x == 0) {
        c->rho = tot.v[0];
        c->rr = tot.v[0];
        c->rr0 = tot.v[0];
        c->iter = 0;
        c->max_it = max_it;
        c->status = 0;
        c->done = 0;
        c->scale = active ? nrm : 0.0;
        c->tol2 = rtol2 * tot.v[0];
        if (!active || !(tot.v[0] > 0.0)) finish_inst(c, 0, n_done);
    }
}

// x64 += |r| * x32 for the instances of the last inner solve.
template <int R>
__global__ void __launch_bounds__(kBlockThreads) k_ir_correct(double *__restrict__ x, const float *__restrict__ x32,
                                                              const InstCtl *__restrict__ ctl,
                                                              const int32_t *__restrict__ tile_inst) {
    const int tile = blockIdx.x;
    const double sc = ctl[tile_inst[tile]].scale;
    if (sc == 0.0) return;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t row = ((int64_t)tile * R + k) * kBlockThreads + threadIdx.x;
        x[row] += sc * (double)x32[row];
    }
}

template <typename T> SellView<T> view(const DevSystem &s);
template <> SellView<double> view<double>(const DevSystem &s) { return {s.n_rows, s.slice_off, s.col, s.val64}; }
template <> SellView<float> view<float>(const DevSystem &s) { return {s.n_rows, s.slice_off, s.col, s.val32}; }

template <int R> cudaError_t cg_init_r(const DevSystem &sys, double rtol2, double atol2, int max_it, int use_active,
                                       cudaStream_t st) {
    k_cg_init<double, R><<<(unsigned)sys.n_tiles, kBlockThreads, 0, st>>>(
        view<double>(sys), sys.bh, sys.x, sys.r, sys.p, sys.partial, sys.ctl, sys.tile_inst, sys.n_done, 1, rtol2,
        atol2, max_it, sys.inst_sums, use_active);
    return cudaGetLastError();
}

template <int R> cudaError_t cg_spmv_r(const DevSystem &sys, int prec, cudaStream_t st) {
    const unsigned g = (unsigned)sys.n_tiles;
    if (prec == 64)
        k_cg_spmv<double, R><<<g, kBlockThreads, 0, st>>>(view<double>(sys), sys.p, sys.q, sys.r, sys.partial, sys.ctl,
                                                          sys.tile_inst, sys.n_done);
    else
        k_cg_spmv<float, R><<<g, kBlockThreads, 0, st>>>(view<float>(sys), sys.p32, sys.q32, sys.r32, sys.partial,
                                                         sys.ctl, sys.tile_inst, sys.n_done);
    return cudaGetLastError();
}

template <int R> cudaError_t cg_update_r(const DevSystem &sys, int prec, cudaStream_t st) {
    const unsigned g = (unsigned)sys.n_tiles;
    if (prec == 64)
        k_cg_update<double, R><<<g, kBlockThreads, 0, st>>>(sys.x, sys.r, sys.p, sys.q, sys.partial, sys.ctl,
                                                            sys.tile_inst, sys.n_done);
    else
        k_cg_update<float, R><<<g, kBlockThreads, 0, st>>>(sys.x32, sys.r32, sys.p32, sys.q32, sys.partial, sys.ctl,
                                                           sys.tile_inst, sys.n_done);
    return cudaGetLastError();
}

template <int R> cudaError_t cg_iter_r(const DevSystem &sys, int prec, cudaStream_t st) {
    cudaError_t e = cg_spmv_r<R>(sys, prec, st);
    return e == cudaSuccess ? cg_update_r<R>(sys, prec, st) : e;
}

}  // namespace

cudaError_t launch_cg_init(const DevSystem &sys, double rtol2, double atol2, int max_it, int use_active,
                           cudaStream_t s) {
    switch (sys.rows_per_thread) {
        case 1: return cg_init_r<1>(sys, rtol2, atol2, max_it, use_active, s);
        case 2: return cg_init_r<2>(sys, rtol2, atol2, max_it, use_active, s);
        case 4: return cg_init_r<4>(sys, rtol2, atol2, max_it, use_active, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cg_spmv(const DevSystem &sys, int prec, cudaStream_t s) {
    switch (sys.rows_per_thread) {
        case 1: return cg_spmv_r<1>(sys, prec, s);
        case 2: return cg_spmv_r<2>(sys, prec, s);
        case 4: return cg_spmv_r<4>(sys, prec, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cg_update(const DevSystem &sys, int prec, cudaStream_t s) {
    switch (sys.rows_per_thread) {
        case 1: return cg_update_r<1>(sys, prec, s);
        case 2: return cg_update_r<2>(sys, prec, s);
        case 4: return cg_update_r<4>(sys, prec, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cg_iteration(const DevSystem &sys, int prec, cudaStream_t s) {
    switch (sys.rows_per_thread) {
        case 1: return cg_iter_r<1>(sys, prec, s);
        case 2: return cg_iter_r<2>(sys, prec, s);
        case 4: return cg_iter_r<4>(sys, prec, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_residual64(const DevSystem &sys, cudaStream_t s) {
    const unsigned g = (unsigned)sys.n_tiles;
    switch (sys.rows_per_thread) {
        case 1: k_residual64<1><<<g, kBlockThreads, 0, s>>>(view<double>(sys), sys.bh, sys.x, sys.dsq, sys.r, sys.partial, sys.ctl, sys.tile_inst, sys.inst_sums); break;
        case 2: k_residual64<2><<<g, kBlockThreads, 0, s>>>(view<double>(sys), sys.bh, sys.x, sys.dsq, sys.r, sys.partial, sys.ctl, sys.tile_inst, sys.inst_sums); break;
        case 4: k_residual64<4><<<g, kBlockThreads, 0, s>>>(view<double>(sys), sys.bh, sys.x, sys.dsq, sys.r, sys.partial, sys.ctl, sys.tile_inst, sys.inst_sums); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_ir_start(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s) {
    const unsigned g = (unsigned)sys.n_tiles;
    switch (sys.rows_per_thread) {
        case 1: k_ir_start<1><<<g, kBlockThreads, 0, s>>>(sys.r, sys.x32, sys.r32, sys.p32, sys.partial, sys.ctl, sys.tile_inst, sys.inst_sums, sys.n_done, rtol2, max_it); break;
        case 2: k_ir_start<2><<<g, kBlockThreads, 0, s>>>(sys.r, sys.x32, sys.r32, sys.p32, sys.partial, sys.ctl, sys.tile_inst, sys.inst_sums, sys.n_done, rtol2, max_it); break;
        case 4: k_ir_start<4><<<g, kBlockThreads, 0, s>>>(sys.r, sys.x32, sys.r32, sys.p32, sys.partial, sys.ctl, sys.tile_inst, sys.inst_sums, sys.n_done, rtol2, max_it); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_ir_correct(const DevSystem &sys, cudaStream_t s) {
    const unsigned g = (unsigned)sys.n_tiles;
    switch (sys.rows_per_thread) {
        case 1: k_ir_correct<1><<<g, kBlockThreads, 0, s>>>(sys.x, sys.x32, sys.ctl, sys.tile_inst); break;
        case 2: k_ir_correct<2><<<g, kBlockThreads, 0, s>>>(sys.x, sys.x32, sys.ctl, sys.tile_inst); break;
        case 4: k_ir_correct<4><<<g, kBlockThreads, 0, s>>>(sys.x, sys.x32, sys.ctl, sys.tile_inst); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_reset_ctl(const DevSystem &sys, cudaStream_t s) {
    return cudaMemsetAsync(sys.n_done, 0, sizeof(int32_t), s);
}

}  // namespace mh
