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
// Work distribution: rows are grouped into tiles of 256*R rows (a 256-thread block runs R
// 32-row slices per warp), tiles never straddle instances, and a host-built block plan gives
// every block a contiguous run of one instance's tiles (about as many blocks as fit on the GPU
// at once).  A block accumulates over its tiles and publishes one partial sum; the last block of
// an instance to arrive (atomic ticket, no spin-wait) sums that instance's partials in a fixed
// order.  The reductions are therefore deterministic, each block pays for one fence and one
// atomic per kernel, and a batch of independent systems shares every launch while each keeps
// its own alpha/beta/convergence (per-instance masks).
#include <cuda_runtime.h>

#include "device_system.hpp"

namespace mh {

namespace {

template <int NV> struct Sums { double v[NV]; };

// Block-wide sum of NV doubles; result valid in thread 0.  Fixed order.
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

struct Plan {
    const int32_t *inst, *tile_begin, *tile_end, *inst_blk;
};

// Publishes this block's partial sums and returns true in every thread of the block that
// arrived last for its instance; that block then holds the instance totals in `tot`
// (thread 0 only).
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
        const unsigned t = atomicAdd(&c->ticket, 1u);
        am_last = (t == (unsigned)(pe - pb) - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    // eight independent accumulators per thread keep eight loads in flight
    constexpr int U = 8;
    double acc[U][NV];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[u][k] = 0.0;
    for (int t0 = pb + threadIdx.x; t0 < pe; t0 += U * blockDim.x) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < pe) {
#pragma unroll
                for (int k = 0; k < NV; ++k) acc[u][k] += __ldcg(&partial[(int64_t)t * 4 + k]);
            }
        }
    }
    Sums<NV> a;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        a.v[k] = 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u) a.v[k] += acc[u][k];
    }
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

__device__ __forceinline__ int64_t slice_of(int tile, int warp, int R, int k) {
    return ((int64_t)tile * kWarpsPerBlock + warp) * R + k;
}

// y = (S^ v)[row] for the R rows this thread owns in `tile`; all loads of the first kJ slots
// of the R slices are issued before any use (2*kJ*R streaming loads and kJ*R gathers in flight).
template <typename T, typename V, int R>
__device__ __forceinline__ void sell_rows(const SellView<T> &A, const V *__restrict__ v, int tile, double (&y)[R]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kJ = 8;
    int64_t off[R];
    int w[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int64_t sl = slice_of(tile, warp, R, k);
        off[k] = A.slice_off[sl];
        w[k] = (int)((A.slice_off[sl + 1] - off[k]) / kSliceRows);
    }
    int32_t cj[R][kJ];
    T vj[R][kJ];
#pragma unroll
    for (int k = 0; k < R; ++k)
#pragma unroll
        for (int j = 0; j < kJ; ++j) {
            const bool in = j < w[k];
            const int64_t slot = off[k] + (int64_t)j * kSliceRows + lane;
            cj[k][j] = in ? ldg_stream(A.col + slot) : 0;
            vj[k][j] = in ? ldg_stream(A.val + slot) : (T)0;
        }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < kJ; ++j) acc += (double)vj[k][j] * (double)v[cj[k][j]];
        for (int j = kJ; j < w[k]; ++j) {
            const int64_t slot = off[k] + (int64_t)j * kSliceRows + lane;
            acc += (double)ldg_stream(A.val + slot) * (double)v[ldg_stream(A.col + slot)];
        }
        y[k] = acc;
    }
}

template <int R> __device__ __forceinline__ int64_t sell_row(int tile, int k) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return slice_of(tile, warp, R, k) * kSliceRows + lane;
}

template <int R> __device__ __forceinline__ int64_t flat_row(int tile, int k) {
    return ((int64_t)tile * R + k) * kBlockThreads + threadIdx.x;
}

// One thread's share of a SELL tile for the pipelined SpMV (R = 1): the first kJ slots of its
// row (column index and value) and the own-row entries of p and r.
template <typename T> struct SpmvStage {
    static constexpr int kJ = 8;
    int64_t off;
    int w;
    int32_t c[kJ];
    T v[kJ];
    T pr, rr;
};

template <typename T>
__device__ __forceinline__ void spmv_stage_load(const SellView<T> &A, const T *__restrict__ p, const T *__restrict__ r,
                                                int tile, SpmvStage<T> &st) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t sl = slice_of(tile, warp, 1, 0);
    st.off = A.slice_off[sl];
    st.w = (int)((A.slice_off[sl + 1] - st.off) / kSliceRows);
#pragma unroll
    for (int j = 0; j < SpmvStage<T>::kJ; ++j) {
        const bool in = j < st.w;
        const int64_t slot = st.off + (int64_t)j * kSliceRows + lane;
        st.c[j] = in ? ldg_stream(A.col + slot) : 0;
        st.v[j] = in ? ldg_stream(A.val + slot) : (T)0;
    }
    const int64_t row = sl * kSliceRows + lane;
    st.pr = p[row];
    st.rr = r[row];
}

// q = S^ p and the three dot products.  Software-pipelined over the block's tiles: the
// indices, values and own-row vector entries of tile t+1 are loaded while the gathers of
// tile t are in flight, so every thread always has a full tile of loads outstanding.
template <typename T, int R>
__global__ void __launch_bounds__(kBlockThreads, sizeof(T) == 4 ? 4 : 3)
    k_cg_spmv(SellView<T> A, const T *__restrict__ p, T *__restrict__ q,
                                                           const T *__restrict__ r, double *__restrict__ partial,
                                                           InstCtl *__restrict__ ctl, Plan plan, int32_t *n_done) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (c->done) return;
    Sums<3> s = {{0.0, 0.0, 0.0}};
    const int tb = plan.tile_begin[blockIdx.x], te = plan.tile_end[blockIdx.x];
    if (R == 1) {
        constexpr int kJ = SpmvStage<T>::kJ;
        const int lane = threadIdx.x & 31;
        SpmvStage<T> st;
        if (tb < te) spmv_stage_load<T>(A, p, r, tb, st);
        for (int tile = tb; tile < te; ++tile) {
            T g[kJ];
#pragma unroll
            for (int j = 0; j < kJ; ++j) g[j] = p[st.c[j]];
            const SpmvStage<T> cur = st;
            if (tile + 1 < te) spmv_stage_load<T>(A, p, r, tile + 1, st);
            double y = 0.0;
#pragma unroll
            for (int j = 0; j < kJ; ++j) y += (double)cur.v[j] * (double)g[j];
            for (int j = kJ; j < cur.w; ++j) {
                const int64_t slot = cur.off + (int64_t)j * kSliceRows + lane;
                y += (double)ldg_stream(A.val + slot) * (double)p[ldg_stream(A.col + slot)];
            }
            q[sell_row<1>(tile, 0)] = (T)y;
            s.v[0] += (double)cur.pr * y;
            s.v[1] += (double)cur.rr * y;
            s.v[2] += y * y;
        }
    } else {
        for (int tile = tb; tile < te; ++tile) {
            double y[R];
            sell_rows<T, T, R>(A, p, tile, y);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int64_t row = sell_row<R>(tile, k);
                q[row] = (T)y[k];
                const double pr = (double)p[row], rr = (double)r[row];
                s.v[0] += pr * y[k];
                s.v[1] += rr * y[k];
                s.v[2] += y[k] * y[k];
            }
        }
    }
    Sums<3> tot;
    if (block_finish<3>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
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
                                                             InstCtl *__restrict__ ctl, Plan plan, int32_t *n_done) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (c->done) return;
    const double alpha = c->alpha, beta = c->beta;
    Sums<1> s = {{0.0}};
    // software-pipelined: the four loads of tile t+1 are issued before tile t is computed
    const int tb = plan.tile_begin[blockIdx.x], te = plan.tile_end[blockIdx.x];
    T pv[R], xv[R], rv[R], qv[R];
    auto load = [&](int tile) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int64_t row = flat_row<R>(tile, k);
            pv[k] = p[row];
            xv[k] = x[row];
            rv[k] = r[row];
            qv[k] = ldg_stream(q + row);
        }
    };
    if (tb < te) load(tb);
    for (int tile = tb; tile < te; ++tile) {
        T cp[R], cx[R], cr[R], cq[R];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            cp[k] = pv[k];
            cx[k] = xv[k];
            cr[k] = rv[k];
            cq[k] = qv[k];
        }
        if (tile + 1 < te) load(tile + 1);
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int64_t row = flat_row<R>(tile, k);
            const double pr = (double)cp[k];
            const double rr = (double)cr[k] - alpha * (double)cq[k];
            x[row] = (T)((double)cx[k] + alpha * pr);
            r[row] = (T)rr;
            p[row] = (T)(rr + beta * pr);
            const double rs = (double)(T)rr;
            s.v[0] += rs * rs;
        }
    }
    Sums<1> tot;
    if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
        const double rr = tot.v[0];
        c->rho = rr;
        c->rr = rr;
        c->iter += 1;
        if (!isfinite(rr)) finish_inst(c, -6, n_done);
        else if (rr <= c->tol2) finish_inst(c, 0, n_done);
        else if (c->iter >= c->max_it) finish_inst(c, 1, n_done);
    }
}

// r = bh - S^ x; p = r; start an FP64 CG run.  tol2 = max(rtol2 * bh.bh, atol2).
// With use_active, instances whose flag inst_sums[kSumStride*i + kSumActive] is 0 are
// marked done at once.
template <int R>
__global__ void __launch_bounds__(kBlockThreads) k_cg_init(SellView<double> A, const double *__restrict__ b,
                                                           const double *__restrict__ x, double *__restrict__ r,
                                                           double *__restrict__ p, double *__restrict__ partial,
                                                           InstCtl *__restrict__ ctl, Plan plan, int32_t *n_done,
                                                           double rtol2, double atol2, int max_it,
                                                           const double *__restrict__ inst_sums, int use_active) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    const bool active = !use_active || inst_sums[kSumStride * inst + kSumActive] != 0.0;
    Sums<2> s = {{0.0, 0.0}};
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        double y[R];
        sell_rows<double, double, R>(A, x, tile, y);
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int64_t row = sell_row<R>(tile, k);
            const double bb = b[row];
            const double rr = bb - y[k];
            r[row] = rr;
            p[row] = rr;
            s.v[0] += rr * rr;
            s.v[1] += bb * bb;
        }
    }
    Sums<2> tot;
    if (block_finish<2>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
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
        c->tol2 = fmax(rtol2 * bb, atol2);
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
                                                              InstCtl *__restrict__ ctl, Plan plan,
                                                              double *__restrict__ inst_sums) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    Sums<4> s = {{0.0, 0.0, 0.0, 0.0}};
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        double y[R];
        sell_rows<double, double, R>(A, x, tile, y);
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int64_t row = sell_row<R>(tile, k);
            const double b = bh[row];
            const double rr = b - y[k];
            r[row] = rr;
            const double d = dsq[row] * dsq[row];
            s.v[0] += rr * rr;
            s.v[1] += d * rr * rr;
            s.v[2] += d * b * b;
            s.v[3] += b * b;
        }
    }
    Sums<4> tot;
    if (block_finish<4>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) inst_sums[kSumStride * inst + k] = tot.v[k];
    }
}

// Starts (keep_p = 0) or continues after a reliable update (keep_p = 1) an FP32 inner solve
// of S^ d = r / |r| for every instance whose outer residual is above its target
// (inst_sums[kSumStride*i + kSumActive] = 1).  On a reliable update the FP32 recursion
// continues from the recomputed FP64 residual and the search direction is kept, rescaled from
// the old normalisation |r_old| to the new |r_new|, so no Krylov information is lost.
// keep_p = 2 (flexible CG) leaves p and the stored (p, q) pair untouched: the next direction
// is made conjugate to them, which needs no common scale.
template <int R>
__global__ void __launch_bounds__(kBlockThreads) k_ir_start(const double *__restrict__ r64, float *__restrict__ x32,
                                                            float *__restrict__ r32, float *__restrict__ p32,
                                                            double *__restrict__ partial, InstCtl *__restrict__ ctl,
                                                            Plan plan, const double *__restrict__ inst_sums,
                                                            int32_t *n_done, double rtol2, int max_it, int keep_p) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    const bool active = inst_sums[kSumStride * inst + kSumActive] != 0.0;
    const double nrm = sqrt(inst_sums[kSumStride * inst + 0]);
    const double inv = (active && nrm > 0.0) ? 1.0 / nrm : 0.0;
    const double ratio = (active && nrm > 0.0) ? c->scale / nrm : 0.0;
    Sums<1> s = {{0.0}};
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int64_t row = flat_row<R>(tile, k);
            const float v = (float)(r64[row] * inv);
            x32[row] = 0.0f;
            r32[row] = v;
            if (keep_p == 0) p32[row] = v;
            else if (keep_p == 1) p32[row] = (float)((double)p32[row] * ratio);
            s.v[0] += (double)v * (double)v;
        }
    }
    Sums<1> tot;
    if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
        c->rho = tot.v[0];
        c->rr = tot.v[0];
        c->rr0 = tot.v[0];
        c->iter = 0;
        c->max_it = max_it;
        c->status = 0;
        c->done = 0;
        c->scale = active ? nrm : 0.0;
        c->tol2 = rtol2 * tot.v[0];
        if (keep_p != 2) c->aux[1] = 0.0;  // flexible CG: no stored direction, restart
        if (!active || !(tot.v[0] > 0.0)) finish_inst(c, 0, n_done);
    }
}

// x64 += |r| * x32 for the instances of the last inner solve.
template <int R>
__global__ void __launch_bounds__(kBlockThreads) k_ir_correct(double *__restrict__ x, const float *__restrict__ x32,
                                                              const InstCtl *__restrict__ ctl, Plan plan) {
    const double sc = ctl[plan.inst[blockIdx.x]].scale;
    if (sc == 0.0) return;
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile)
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int64_t row = flat_row<R>(tile, k);
            x[row] += sc * (double)x32[row];
        }
}

template <typename T> SellView<T> view(const DevSystem &s);
template <> SellView<double> view<double>(const DevSystem &s) { return {s.n_rows, s.slice_off, s.col, s.val64}; }
template <> SellView<float> view<float>(const DevSystem &s) { return {s.n_rows, s.slice_off, s.col, s.val32}; }

// plan 0 serves the FP64 kernels, plan 1 the FP32 ones
Plan plan_of(const DevSystem &s, int prec) {
    const DevPlan &p = s.plan[prec == 64 ? 0 : 1];
    return {p.blk_inst, p.tile_begin, p.tile_end, p.inst_blk};
}
unsigned grid_of(const DevSystem &s, int prec) { return (unsigned)s.plan[prec == 64 ? 0 : 1].n_blocks; }

template <int R> cudaError_t cg_init_r(const DevSystem &sys, double rtol2, double atol2, int max_it, int use_active,
                                       cudaStream_t st) {
    k_cg_init<R><<<grid_of(sys, 64), kBlockThreads, 0, st>>>(view<double>(sys), sys.bh, sys.x, sys.r, sys.p,
                                                              sys.partial, sys.ctl, plan_of(sys, 64), sys.n_done,
                                                              rtol2, atol2, max_it, sys.inst_sums, use_active);
    return cudaGetLastError();
}

template <int R> cudaError_t cg_spmv_r(const DevSystem &sys, int prec, cudaStream_t st) {
    const unsigned g = grid_of(sys, prec);
    if (prec == 64)
        k_cg_spmv<double, R><<<g, kBlockThreads, 0, st>>>(view<double>(sys), sys.p, sys.q, sys.r, sys.partial, sys.ctl,
                                                          plan_of(sys, 64), sys.n_done);
    else
        k_cg_spmv<float, R><<<g, kBlockThreads, 0, st>>>(view<float>(sys), sys.p32, sys.q32, sys.r32, sys.partial,
                                                         sys.ctl, plan_of(sys, 32), sys.n_done);
    return cudaGetLastError();
}

template <int R> cudaError_t cg_update_r(const DevSystem &sys, int prec, cudaStream_t st) {
    const unsigned g = grid_of(sys, prec);
    if (prec == 64)
        k_cg_update<double, R><<<g, kBlockThreads, 0, st>>>(sys.x, sys.r, sys.p, sys.q, sys.partial, sys.ctl,
                                                            plan_of(sys, 64), sys.n_done);
    else
        k_cg_update<float, R><<<g, kBlockThreads, 0, st>>>(sys.x32, sys.r32, sys.p32, sys.q32, sys.partial, sys.ctl,
                                                           plan_of(sys, 32), sys.n_done);
    return cudaGetLastError();
}

template <int R> cudaError_t residual_r(const DevSystem &sys, cudaStream_t st) {
    k_residual64<R><<<grid_of(sys, 64), kBlockThreads, 0, st>>>(view<double>(sys), sys.bh, sys.x, sys.dsq, sys.r,
                                                                 sys.partial, sys.ctl, plan_of(sys, 64),
                                                                 sys.inst_sums);
    return cudaGetLastError();
}

template <int R> cudaError_t ir_start_r(const DevSystem &sys, double rtol2, int max_it, int keep_p, cudaStream_t st) {
    k_ir_start<R><<<grid_of(sys, 32), kBlockThreads, 0, st>>>(sys.r, sys.x32, sys.r32, sys.p32, sys.partial, sys.ctl,
                                                               plan_of(sys, 32), sys.inst_sums, sys.n_done, rtol2,
                                                               max_it, keep_p);
    return cudaGetLastError();
}

template <int R> cudaError_t ir_correct_r(const DevSystem &sys, cudaStream_t st) {
    k_ir_correct<R><<<grid_of(sys, 32), kBlockThreads, 0, st>>>(sys.x, sys.x32, sys.ctl, plan_of(sys, 32));
    return cudaGetLastError();
}

}  // namespace

#define MH_BY_R(CALL)                                      \
    switch (sys.rows_per_thread) {                         \
        case 1: return CALL(1);                            \
        case 2: return CALL(2);                            \
        case 4: return CALL(4);                            \
        default: return cudaErrorInvalidValue;             \
    }

cudaError_t launch_cg_init(const DevSystem &sys, double rtol2, double atol2, int max_it, int use_active,
                           cudaStream_t s) {
#define C_(R) cg_init_r<R>(sys, rtol2, atol2, max_it, use_active, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_cg_spmv(const DevSystem &sys, int prec, cudaStream_t s) {
#define C_(R) cg_spmv_r<R>(sys, prec, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_cg_update(const DevSystem &sys, int prec, cudaStream_t s) {
#define C_(R) cg_update_r<R>(sys, prec, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_cg_iteration(const DevSystem &sys, int prec, cudaStream_t s) {
    cudaError_t e = launch_cg_spmv(sys, prec, s);
    return e == cudaSuccess ? launch_cg_update(sys, prec, s) : e;
}

cudaError_t launch_residual64(const DevSystem &sys, cudaStream_t s) {
#define C_(R) residual_r<R>(sys, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_ir_start(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s) {
#define C_(R) ir_start_r<R>(sys, rtol2, max_it, 0, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_ir_replace(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s) {
#define C_(R) ir_start_r<R>(sys, rtol2, max_it, 1, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_ir_continue(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s) {
#define C_(R) ir_start_r<R>(sys, rtol2, max_it, 2, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_ir_correct(const DevSystem &sys, cudaStream_t s) {
#define C_(R) ir_correct_r<R>(sys, s)
    MH_BY_R(C_)
#undef C_
}

cudaError_t launch_reset_ctl(const DevSystem &sys, cudaStream_t s) {
    return cudaMemsetAsync(sys.n_done, 0, sizeof(int32_t), s);
}

// Loop control of a conditional WHILE graph node (the device-side Krylov loop): the body runs
// while some instance is not done and fewer than loop[1] bodies have run.  loop[0] counts the
// bodies; the count bounds the loop whatever the kernels of the body do.
__global__ void k_loop_init(cudaGraphConditionalHandle hnd, int32_t *__restrict__ loop,
                            const int32_t *__restrict__ n_done, int32_t n_inst) {
    loop[0] = 0;
    cudaGraphSetConditional(hnd, (*n_done < n_inst && loop[1] > 0) ? 1u : 0u);
}

__global__ void k_loop_next(cudaGraphConditionalHandle hnd, int32_t *__restrict__ loop,
                            const int32_t *__restrict__ n_done, int32_t n_inst) {
    const int32_t c = loop[0] + 1;
    loop[0] = c;
    cudaGraphSetConditional(hnd, (*n_done < n_inst && c < loop[1]) ? 1u : 0u);
}

cudaError_t launch_loop_init(const DevSystem &sys, cudaGraphConditionalHandle hnd, int32_t *loop, cudaStream_t s) {
    k_loop_init<<<1, 1, 0, s>>>(hnd, loop, sys.n_done, sys.n_inst);
    return cudaGetLastError();
}

cudaError_t launch_loop_next(const DevSystem &sys, cudaGraphConditionalHandle hnd, int32_t *loop, cudaStream_t s) {
    k_loop_next<<<1, 1, 0, s>>>(hnd, loop, sys.n_done, sys.n_inst);
    return cudaGetLastError();
}

int krylov_target_blocks(int rows_per_thread, int prec) {
    int dev = 0, sms = 148, per_sm = 4;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) {
        int a = 0;
        cudaError_t e = cudaErrorInvalidValue;
        const bool f64 = prec == 64;
        switch (rows_per_thread) {
            case 1:
                e = f64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cg_spmv<double, 1>, kBlockThreads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cg_spmv<float, 1>, kBlockThreads, 0);
                break;
            case 2:
                e = f64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cg_spmv<double, 2>, kBlockThreads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cg_spmv<float, 2>, kBlockThreads, 0);
                break;
            default:
                e = f64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cg_spmv<double, 4>, kBlockThreads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cg_spmv<float, 4>, kBlockThreads, 0);
                break;
        }
        if (e == cudaSuccess && a > 0) per_sm = a;
        else cudaGetLastError();
    } else {
        cudaGetLastError();
        sms = 148;
    }
    const char *env = getenv(prec == 64 ? "MH_BLOCKS_PER_SM_64" : "MH_BLOCKS_PER_SM_32");
    if (env) {
        int v = atoi(env);
        if (v >= 1 && v <= 32) per_sm = v;
    }
    return sms * per_sm;
}

}  // namespace mh
