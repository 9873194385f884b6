// K7: learned preconditioner (message passing over the edge system) and the flexible-CG and
// Chebyshev-Jacobi kernels that use it.  No counterpart in the reference, which preconditions
// with PETSc ILU (src/la/solve.cc:370); this is the preconditioner of the FCG solver.
//
// Network, applied to a residual r of the Jacobi-scaled edge system S^ (unit diagonal):
//   h0_i = (r_i, 0, 0, 0);  per layer l = 0..2:
//     a = S^ h^l                         (4 channels, SELL SpMV with float4 gathers)
//     s_i = W1 [h^l_i ; a_i] + b1        (8 -> 32)   \  tensor cores: mma.sync m16n8k16,
//     o_i = W2 relu(s_i) + b2            (32 -> 4)   /  bf16 operands, fp32 accumulation
//     h^{l+1}_i = h^l_i + o_i
//   z_i = h3_i[0].
// With W2 = b2 = 0 it is the identity (Jacobi), the starting point of training.  Training runs
// an FP32 CUDA-core forward that rounds the same operands to bf16 (so it matches the tensor-core
// inference), an FP32 backward, the energy-norm loss (z-e)'S^(z-e)/(e'S^e) and Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_system.hpp"
#include "learned.hpp"

namespace mh {

namespace {

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

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
template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(kBlockThreads)
    k_nn_layer(SellView<float> A, const float *__restrict__ r, const float4 *__restrict__ h_in,
               float4 *__restrict__ h_out, float *__restrict__ z_out, float4 *__restrict__ a_out,
               NnLayerView wl, const float *__restrict__ q_old, double *__restrict__ partial,
               InstCtl *__restrict__ ctl, Plan plan, int32_t *n_done, int skip_done,
               const int32_t *__restrict__ row_edge) {
    const int inst = plan.inst[blockIdx.x];
    InstCtl *c = ctl + inst;
    if (skip_done && c->done) return;
    __shared__ float su[kWarpsPerBlock][kSliceRows][8];
    __shared__ float so[kWarpsPerBlock][kSliceRows][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    // B fragments: W1 (32x8, k padded to 16) as 4 n-tiles; W2 (4x32, n padded to 8) as 2 k-steps
    uint32_t b1[4], b2[2][2];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) b1[nt] = wl.w1b[(8 * nt + g) * 4 + t];
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
        b2[ks][0] = g < 4 ? wl.w2b[g * 16 + ks * 8 + t] : 0u;
        b2[ks][1] = g < 4 ? wl.w2b[g * 16 + ks * 8 + 4 + t] : 0u;
    }
    float bias1[4][2];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        bias1[nt][0] = wl.b1[8 * nt + 2 * t];
        bias1[nt][1] = wl.b1[8 * nt + 2 * t + 1];
    }
    const float4 bias2 = make_float4(wl.b2[0], wl.b2[1], wl.b2[2], wl.b2[3]);
    // the network sees r / |r| (its training pairs are normalised the same way) and its output
    // is scaled back by |r|, so the preconditioner is positively homogeneous
    const double rn = sqrt(c->rr);
    const float inv = (FIRST && rn > 0.0) ? (float)(1.0 / rn) : 1.f;
    double zq = 0.0;
    for (int tile = plan.tile_begin[blockIdx.x]; tile < plan.tile_end[blockIdx.x]; ++tile) {
        const int64_t sl = (int64_t)tile * kWarpsPerBlock + warp;
        const int64_t row = sl * kSliceRows + lane;
        const float4 hi = FIRST ? make_float4(r[row] * inv, 0.f, 0.f, 0.f) : h_in[row];
        float4 ai = aggregate<FIRST>(A, r, h_in, sl, lane);
        if (FIRST) ai.x *= inv;
        if (a_out) a_out[row] = ai;
        su[warp][lane][0] = hi.x; su[warp][lane][1] = hi.y; su[warp][lane][2] = hi.z; su[warp][lane][3] = hi.w;
        su[warp][lane][4] = ai.x; su[warp][lane][5] = ai.y; su[warp][lane][6] = ai.z; su[warp][lane][7] = ai.w;
        __syncwarp();
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int r0 = 16 * half + g, r1 = r0 + 8;
            uint32_t a[4];
            a[0] = pack_bf16(su[warp][r0][2 * t], su[warp][r0][2 * t + 1]);
            a[1] = pack_bf16(su[warp][r1][2 * t], su[warp][r1][2 * t + 1]);
            a[2] = 0u;  // k = 8..15 is padding
            a[3] = 0u;
            float hid[4][4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                hid[nt][0] = bias1[nt][0];
                hid[nt][1] = bias1[nt][1];
                hid[nt][2] = bias1[nt][0];
                hid[nt][3] = bias1[nt][1];
                mma_bf16(hid[nt], a, b1[nt], 0u);
            }
            float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                uint32_t a2[4];
                a2[0] = pack_bf16(fmaxf(hid[2 * ks][0], 0.f), fmaxf(hid[2 * ks][1], 0.f));
                a2[1] = pack_bf16(fmaxf(hid[2 * ks][2], 0.f), fmaxf(hid[2 * ks][3], 0.f));
                a2[2] = pack_bf16(fmaxf(hid[2 * ks + 1][0], 0.f), fmaxf(hid[2 * ks + 1][1], 0.f));
                a2[3] = pack_bf16(fmaxf(hid[2 * ks + 1][2], 0.f), fmaxf(hid[2 * ks + 1][3], 0.f));
                mma_bf16(o, a2, b2[ks][0], b2[ks][1]);
            }
            if (t < 2) {  // output columns 2t, 2t+1 < 4 are the real ones
                so[warp][r0][2 * t] = o[0];
                so[warp][r0][2 * t + 1] = o[1];
                so[warp][r1][2 * t] = o[2];
                so[warp][r1][2 * t + 1] = o[3];
            }
        }
        __syncwarp();
        float4 ho;
        ho.x = hi.x + so[warp][lane][0] + bias2.x;
        ho.y = hi.y + so[warp][lane][1] + bias2.y;
        ho.z = hi.z + so[warp][lane][2] + bias2.z;
        ho.w = hi.w + so[warp][lane][3] + bias2.w;
        if (row_edge[row] < 0) ho = make_float4(0.f, 0.f, 0.f, 0.f);  // padding row: stays zero
        if (LAST) {
            const float zv = (float)((double)ho.x * rn);
            z_out[row] = zv;
            if (q_old) zq += (double)zv * (double)q_old[row];
        } else {
            h_out[row] = ho;
        }
        __syncwarp();
    }
    if (LAST && partial) {
        Sums<1> s = {{zq}};
        Sums<1> tot;
        if (block_finish<1>(s, partial, c, plan, inst, tot) && threadIdx.x == 0) {
            // flexible CG (one stored direction): beta = z.q_old / (p.q)_old, 0 on a restart
            c->beta = (c->aux[1] != 0.0 && c->aux[0] != 0.0) ? tot.v[0] / c->aux[0] : 0.0;
        }
    }
}

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

// ---- training -------------------------------------------------------------------------
// h0 = (r, 0, 0, 0)
__global__ void k_nn_h0(const float *__restrict__ r, float4 *__restrict__ h, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) h[i] = make_float4(r[i], 0.f, 0.f, 0.f);
}

// z = h.x
__global__ void k_nn_extract(const float4 *__restrict__ h, float *__restrict__ z, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = h[i].x;
}

// Energy-norm loss of one pair: Sz = S^ z, g = 2 (Sz - r) / (e.r) as a float4 (channel 0),
// partial sums {(z-e).(Sz-r), e.r}.
__global__ void k_nn_loss(SellView<float> A, int64_t n_rows, const float *__restrict__ z, const float *__restrict__ r,
                          const float *__restrict__ e, double er, float4 *__restrict__ g, double *__restrict__ loss) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (row < n_rows) {
        const int64_t sl = row / kSliceRows;
        const int lane = (int)(row % kSliceRows);
        const float4 sz = aggregate<true>(A, z, nullptr, sl, lane);
        const double res = (double)sz.x - (double)r[row];
        g[row] = make_float4((float)(2.0 * res / er), 0.f, 0.f, 0.f);
        l = ((double)z[row] - (double)e[row]) * res;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / er);
}

// Backward of one layer, node-local part: given g' = dL/dh^{l+1}, recompute the layer from
// (h^l, a^l), accumulate the weight gradients, write g_a = dL/da and g_h = g' + dL/dh|direct.
// The aggregation's contribution S^ g_a is added by k_nn_bwd_spmv.
__global__ void __launch_bounds__(128)
    k_nn_bwd_local(int64_t n, const float4 *__restrict__ h, const float4 *__restrict__ a,
                   const float4 *__restrict__ gout, const float *__restrict__ w, float4 *__restrict__ g_a,
                   float4 *__restrict__ g_h, float *__restrict__ grad) {
    __shared__ float sg[kNnPerLayer];
    for (int k = threadIdx.x; k < kNnPerLayer; k += blockDim.x) sg[k] = 0.f;
    __syncthreads();
    const float *W1 = w, *b1 = w + kNnH * 8, *W2 = w + kNnH * 8 + kNnH;
    float *gW1 = sg, *gb1 = sg + kNnH * 8, *gW2 = sg + kNnH * 8 + kNnH, *gb2 = gW2 + 4 * kNnH;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    float u[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float go[4] = {0.f, 0.f, 0.f, 0.f};
    if (active) {
        const float4 hi = h[i], ai = a[i], gi = gout[i];
        u[0] = bf16r(hi.x); u[1] = bf16r(hi.y); u[2] = bf16r(hi.z); u[3] = bf16r(hi.w);
        u[4] = bf16r(ai.x); u[5] = bf16r(ai.y); u[6] = bf16r(ai.z); u[7] = bf16r(ai.w);
        go[0] = gi.x; go[1] = gi.y; go[2] = gi.z; go[3] = gi.w;
    }
    float gu[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < kNnH; ++j) {
        float s = b1[j];
#pragma unroll
        for (int k = 0; k < 8; ++k) s += bf16r(W1[j * 8 + k]) * u[k];
        const float hid = bf16r(fmaxf(s, 0.f));
        float ghid = 0.f;
#pragma unroll
        for (int o = 0; o < 4; ++o) ghid += bf16r(W2[o * kNnH + j]) * go[o];
        const float gs = s > 0.f ? ghid : 0.f;
        // weight gradients, reduced over the warp before one shared atomic per warp
        float v;
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            v = go[o] * hid;
            for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
            if (lane == 0) atomicAdd(&gW2[o * kNnH + j], v);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v = gs * u[k];
            for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
            if (lane == 0) atomicAdd(&gW1[j * 8 + k], v);
            gu[k] += bf16r(W1[j * 8 + k]) * gs;
        }
        v = gs;
        for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
        if (lane == 0) atomicAdd(&gb1[j], v);
    }
#pragma unroll
    for (int o = 0; o < 4; ++o) {
        float v = go[o];
        for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
        if (lane == 0) atomicAdd(&gb2[o], v);
    }
    if (active) {
        g_a[i] = make_float4(gu[4], gu[5], gu[6], gu[7]);
        g_h[i] = make_float4(go[0] + gu[0], go[1] + gu[1], go[2] + gu[2], go[3] + gu[3]);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kNnPerLayer; k += blockDim.x) atomicAdd(&grad[k], sg[k]);
}

// g_h += S^ g_a (S^ symmetric)
__global__ void k_nn_bwd_spmv(SellView<float> A, int64_t n_rows, const float4 *__restrict__ g_a,
                              float4 *__restrict__ g_h) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    const int64_t sl = row / kSliceRows;
    const int lane = (int)(row % kSliceRows);
    const float4 s = aggregate<false>(A, nullptr, g_a, sl, lane);
    float4 v = g_h[row];
    v.x += s.x; v.y += s.y; v.z += s.z; v.w += s.w;
    g_h[row] = v;
}

// Training forward on CUDA cores, numerically the tensor-core layer: bf16 operands, fp32 sums.
__global__ void k_nn_fwd_train(int64_t n, const float4 *__restrict__ h, const float4 *__restrict__ a,
                               const float *__restrict__ w, float4 *__restrict__ h_out,
                               const int32_t *__restrict__ row_edge) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (row_edge[i] < 0) {  // padding row: stays zero
        h_out[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float *W1 = w, *b1 = w + kNnH * 8, *W2 = w + kNnH * 8 + kNnH, *b2 = W2 + 4 * kNnH;
    const float4 hi = h[i], ai = a[i];
    const float u[8] = {bf16r(hi.x), bf16r(hi.y), bf16r(hi.z), bf16r(hi.w),
                        bf16r(ai.x), bf16r(ai.y), bf16r(ai.z), bf16r(ai.w)};
    float o[4] = {0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < kNnH; ++j) {
        float s = b1[j];
#pragma unroll
        for (int k = 0; k < 8; ++k) s += bf16r(W1[j * 8 + k]) * u[k];
        const float hid = bf16r(fmaxf(s, 0.f));
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] += bf16r(W2[q * kNnH + j]) * hid;
    }
    h_out[i] = make_float4(hi.x + o[0] + b2[0], hi.y + o[1] + b2[1], hi.z + o[2] + b2[2], hi.w + o[3] + b2[3]);
}

// a = S^ h (float4) for the training forward
__global__ void k_nn_aggregate(SellView<float> A, int64_t n_rows, const float4 *__restrict__ h,
                               float4 *__restrict__ a) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    a[row] = aggregate<false>(A, nullptr, h, row / kSliceRows, (int)(row % kSliceRows));
}

// Adam on the fp32 master weights, then the bf16 fragments of W1 and W2 for inference.
// Without train_bias the biases b1, b2 stay zero: the network is then positively homogeneous
// (NN(c r) = c NN(r) for c > 0) and maps a residual that vanishes around a row to zero there.
__global__ void k_nn_adam(float *w, float *m, float *v, const float *grad, int n, float lr, float b1, float b2,
                          float eps, float bc1, float bc2, float scale, int train_bias) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = i % kNnPerLayer;
    const bool bias = (k >= kNnH * 8 && k < kNnH * 9) || k >= kNnH * 9 + 4 * kNnH;
    if (bias && !train_bias) return;
    const float g = grad[i] * scale;
    m[i] = b1 * m[i] + (1.f - b1) * g;
    v[i] = b2 * v[i] + (1.f - b2) * g * g;
    w[i] -= lr * (m[i] / bc1) / (sqrtf(v[i] / bc2) + eps);
}

__global__ void k_nn_pack(const float *w, uint32_t *wb) {
    // per layer: W1 (32 x 8) -> 128 words, W2 (4 x 32) -> 64 words
    const int l = blockIdx.x, t = threadIdx.x;
    const float *W1 = w + l * kNnPerLayer, *W2 = W1 + kNnH * 8 + kNnH;
    uint32_t *o = wb + l * kNnPackedPerLayer;
    if (t < 128) o[t] = pack_bf16(W1[2 * t], W1[2 * t + 1]);
    if (t < 64) o[128 + t] = pack_bf16(W2[2 * t], W2[2 * t + 1]);
}

// Training pair from a snapshot of the plain solver: e = x* - x_s, r = r_s (FP32), and
// acc += {r.r, e.r}.
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

NnLayerView nn_layer_view(const float *w, const uint32_t *wb, int l) {
    NnLayerView v;
    v.w1b = wb + l * kNnPackedPerLayer;
    v.w2b = wb + l * kNnPackedPerLayer + 128;
    v.b1 = w + l * kNnPerLayer + kNnH * 8;
    v.b2 = w + l * kNnPerLayer + kNnH * 8 + kNnH + 4 * kNnH;
    return v;
}

cudaError_t launch_nn_pack(const float *w, uint32_t *wb, cudaStream_t s) {
    k_nn_pack<<<kNnLayers, 128, 0, s>>>(w, wb);
    return cudaGetLastError();
}

// z = NN(r) on the FP32 inner vectors; with q_old the last layer reduces z.q_old -> beta.
cudaError_t launch_nn_apply(const DevSystem &sys, const float *w, const uint32_t *wb, const float *r, float4 *h0,
                            float4 *h1, float *z, const float *q_old, cudaStream_t s) {
    if (sys.rows_per_thread != 1) return cudaErrorInvalidValue;  // tiles of 256 rows
    const SellView<float> A = {sys.n_rows, sys.slice_off, sys.col, sys.val32};
    const unsigned g = (unsigned)sys.plan[1].n_blocks;
    const Plan p = plan32(sys);
    k_nn_layer<true, false><<<g, kBlockThreads, 0, s>>>(A, r, nullptr, h0, nullptr, nullptr, nn_layer_view(w, wb, 0),
                                                         nullptr, nullptr, sys.ctl, p, sys.n_done, 1, sys.row_edge);
    k_nn_layer<false, false><<<g, kBlockThreads, 0, s>>>(A, nullptr, h0, h1, nullptr, nullptr,
                                                          nn_layer_view(w, wb, 1), nullptr, nullptr, sys.ctl, p,
                                                          sys.n_done, 1, sys.row_edge);
    k_nn_layer<false, true><<<g, kBlockThreads, 0, s>>>(A, nullptr, h1, nullptr, z, nullptr, nn_layer_view(w, wb, 2),
                                                         q_old, q_old ? sys.partial : nullptr, sys.ctl, p, sys.n_done,
                                                         1, sys.row_edge);
    return cudaGetLastError();
}

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

// One training pass over one pair: forward (storing h^l, a^l), loss, backward; gradients are
// added to grad[kNnParams] and the loss to *loss.
cudaError_t launch_nn_train_pair(const DevSystem &sys, const float *w, const float *r, const float *e, double er,
                                 NnTrainBuffers &b, float *grad, double *loss, cudaStream_t s) {
    const SellView<float> A = {sys.n_rows, sys.slice_off, sys.col, sys.val32};
    const int64_t n = sys.n_rows;
    const unsigned g = blocks_for(n, 256);
    k_nn_h0<<<g, 256, 0, s>>>(r, b.h[0], n);
    for (int l = 0; l < kNnLayers; ++l) {
        k_nn_aggregate<<<g, 256, 0, s>>>(A, n, b.h[l], b.a[l]);
        k_nn_fwd_train<<<g, 256, 0, s>>>(n, b.h[l], b.a[l], w + l * kNnPerLayer, b.h[l + 1], sys.row_edge);
    }
    // z = h3.x (strided view copied into a scalar vector)
    k_nn_extract<<<g, 256, 0, s>>>(b.h[kNnLayers], b.z, n);
    k_nn_loss<<<g, 256, 0, s>>>(A, n, b.z, r, e, er, b.g[0], loss);
    for (int l = kNnLayers - 1; l >= 0; --l) {
        float4 *gin = b.g[(kNnLayers - 1 - l) % 2], *gout = b.g[(kNnLayers - l) % 2];
        k_nn_bwd_local<<<blocks_for(n, 128), 128, 0, s>>>(n, b.h[l], b.a[l], gin, w + l * kNnPerLayer, b.ga, gout,
                                                           grad + l * kNnPerLayer);
        k_nn_bwd_spmv<<<g, 256, 0, s>>>(A, n, b.ga, gout);
    }
    return cudaGetLastError();
}

cudaError_t launch_nn_adam(float *w, float *m, float *v, const float *grad, int step, float lr, float scale,
                           int train_bias, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    k_nn_adam<<<blocks_for(kNnParams, 256), 256, 0, s>>>(w, m, v, grad, kNnParams, lr, b1, b2, 1e-8f, bc1, bc2, scale,
                                                          train_bias);
    return cudaGetLastError();
}

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
