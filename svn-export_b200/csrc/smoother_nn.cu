// Learned smoother: a message-passing network over the edge system that gives every row a
// weight w_i of the multigrid's fine-level smoother (Chebyshev on diag(w) S^ instead of S^), and
// the kernels that train it.  No counterpart in the reference, which preconditions the Schur
// system with PETSc ILU (src/la/solve.cc:370).
//
// Network (per row i of the Jacobi-scaled S^, off-diagonal o_ij):
//   x_i (8 features) = 1, sum|o_ij|, max|o_ij|, sum o_ij, sum max(o_ij, 0), nnz(o_i.)/8,
//                      sum o_ij^2, [no off-diagonal]
//   h0 = relu(W0 x + b0)                      8 -> 32
//   l = 1..3: a = A h,  A_ij = |o_ij|         message passing (one warp per row, lane = channel)
//             u = W_l [h; a] + b_l            64 -> 32: tensor cores, mma.sync m16n8k16 bf16
//             h = h + relu(u)                                 operands, fp32 accumulation
//   z = w_out . h + b_out,  w = exp(ln2 tanh z)      w in [1/2, 2]; w_out = b_out = 0: w = 1
// The network reads the matrix only (not the residual), so the preconditioner it configures is
// a fixed linear SPD operator during a solve: flexible CG keeps its guarantees.
//
// Training (the host loop in mh_handle.cpp) minimises the energy-norm error of the V-cycle on
// residual/error pairs of the plain solver; the gradient with respect to w comes from the
// cycle's adjoint (smoother_grad_w here), the gradient with respect to the parameters from the
// backward kernels below (FP32 CUDA cores, bf16 roundings passed straight through), checked
// against a NumPy restatement of the network.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_system.hpp"
#include "smoother_nn.hpp"

namespace mh {

namespace {

constexpr float kOutC = 0.69314718055994531f;  // ln 2

__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SELL row access of the solver's FP32 matrix (unit diagonal after scaling)
struct Sell {
    const int64_t *off;
    const int32_t *col;
    const float *val;
};

__device__ __forceinline__ void sell_row(const Sell &A, int64_t i, int64_t &base, int &w, int &ln) {
    const int64_t sl = i / kSliceRows;
    ln = (int)(i - sl * kSliceRows);
    base = A.off[sl];
    w = (int)((A.off[sl + 1] - base) / kSliceRows);
}

// ---- features ----------------------------------------------------------------------------
__global__ void k_sn_features(int64_t n, Sell A, const int32_t *__restrict__ row_edge, float *__restrict__ x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s1 = 0.f, mx = 0.f, s3 = 0.f, s4 = 0.f, s6 = 0.f;
    int cnt = 0;
    if (row_edge[i] >= 0) {
        int64_t base;
        int w, ln;
        sell_row(A, i, base, w, ln);
        for (int j = 0; j < w; ++j) {
            const int64_t slot = base + (int64_t)j * kSliceRows + ln;
            const int32_t c = A.col[slot];
            const float v = A.val[slot];
            if (c == (int32_t)i || v == 0.f) continue;
            s1 += fabsf(v);
            mx = fmaxf(mx, fabsf(v));
            s3 += v;
            s4 += fmaxf(v, 0.f);
            s6 += v * v;
            ++cnt;
        }
    }
    float *xi = x + i * kSnF;
    xi[0] = 1.f;
    xi[1] = s1;
    xi[2] = mx;
    xi[3] = s3;
    xi[4] = s4;
    xi[5] = cnt * 0.125f;
    xi[6] = s6;
    xi[7] = cnt == 0 ? 1.f : 0.f;
}

// ---- forward -------------------------------------------------------------------------------
__global__ void k_sn_layer0(int64_t n, const float *__restrict__ x, const float *__restrict__ p,
                            float *__restrict__ u0, float *__restrict__ h0) {
    __shared__ float sw[kSnW * kSnF + kSnW];
    for (int k = threadIdx.x; k < kSnW * kSnF + kSnW; k += blockDim.x)
        sw[k] = k < kSnW * kSnF ? bfr(p[kSnOffW0 + k]) : p[kSnOffB0 + k - kSnW * kSnF];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xi[kSnF];
#pragma unroll
    for (int k = 0; k < kSnF; ++k) xi[k] = bfr(x[i * kSnF + k]);
#pragma unroll 4
    for (int o = 0; o < kSnW; ++o) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < kSnF; ++k) acc += xi[k] * sw[o * kSnF + k];
        acc += sw[kSnW * kSnF + o];
        if (u0) u0[i * kSnW + o] = acc;
        h0[i * kSnW + o] = fmaxf(acc, 0.f);
    }
}

// out[i][c] (+)= sum_{j != i} |o_ij| h[j][c]: one warp per row, lane = channel; the row's slots
// are loaded by the lanes and broadcast
template <bool ACC>
__global__ void __launch_bounds__(256) k_sn_aggregate(int64_t n, Sell A, const float *__restrict__ h,
                                                      float *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    int64_t base;
    int w, ln;
    sell_row(A, i, base, w, ln);
    float acc = 0.f;
    for (int j0 = 0; j0 < w; j0 += 32) {
        int32_t c = -1;
        float v = 0.f;
        if (j0 + lane < w) {
            const int64_t slot = base + (int64_t)(j0 + lane) * kSliceRows + ln;
            c = A.col[slot];
            v = fabsf(A.val[slot]);
        }
        const int m = min(32, w - j0);
        for (int k = 0; k < m; ++k) {
            const int32_t ck = __shfl_sync(0xffffffffu, c, k);
            const float vk = __shfl_sync(0xffffffffu, v, k);
            if (ck != (int32_t)i && vk != 0.f) acc += vk * h[(int64_t)ck * kSnW + lane];
        }
    }
    if (ACC) out[i * kSnW + lane] += acc;
    else out[i * kSnW + lane] = acc;
}

// u = W [h; a] + b, h_out = h + relu(u) for 16 rows per warp on the tensor cores
__global__ void __launch_bounds__(256) k_sn_mlp(int64_t n, const float *__restrict__ h, const float *__restrict__ a,
                                                const float *__restrict__ W, const float *__restrict__ b,
                                                float *__restrict__ u_out, float *__restrict__ h_out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int64_t r0 = ((int64_t)blockIdx.x * 8 + warp) * 16;
    if (r0 >= n) return;
    // B fragments of W^T (K = 64 inputs, N = 32 outputs): 4 k-steps x 4 n-tiles
    uint32_t bw[4][4][2];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const float *wr = W + (8 * nt + g) * (2 * kSnW) + 16 * ks + 2 * t;
            bw[ks][nt][0] = pack2(wr[0], wr[1]);
            bw[ks][nt][1] = pack2(wr[8], wr[9]);
        }
    float acc[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
    const int64_t ra = r0 + g, rb = r0 + g + 8;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        // inputs 16 ks .. 16 ks + 15: h for ks < 2, a for ks >= 2
        const float *src = ks < 2 ? h : a;
        const int k0 = (ks & 1) * 16 + 2 * t;
        uint32_t af[4];
        af[0] = pack2(src[ra * kSnW + k0], src[ra * kSnW + k0 + 1]);
        af[1] = pack2(src[rb * kSnW + k0], src[rb * kSnW + k0 + 1]);
        af[2] = pack2(src[ra * kSnW + k0 + 8], src[ra * kSnW + k0 + 9]);
        af[3] = pack2(src[rb * kSnW + k0 + 8], src[rb * kSnW + k0 + 9]);
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma16816(acc[nt], af, bw[ks][nt][0], bw[ks][nt][1]);
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const int o = 8 * nt + 2 * t;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t row = q < 2 ? ra : rb;
            const int oc = o + (q & 1);
            const float u = acc[nt][q] + b[oc];
            if (u_out) u_out[row * kSnW + oc] = u;
            h_out[row * kSnW + oc] = h[row * kSnW + oc] + fmaxf(u, 0.f);
        }
    }
}

// z = w_out . h + b_out, w = exp(ln2 tanh z) (1 on padding rows): one warp per row, the 32
// channels summed by shuffles in a fixed order
__global__ void __launch_bounds__(256) k_sn_out(int64_t n, const float *__restrict__ h, const float *__restrict__ p,
                                                const int32_t *__restrict__ row_edge, float *__restrict__ z,
                                                float *__restrict__ w) {
    const int64_t i = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    float acc = h[i * kSnW + lane] * p[kSnOffWout + lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane != 0) return;
    acc += p[kSnOffBout];
    if (z) z[i] = acc;
    w[i] = row_edge[i] >= 0 ? expf(kOutC * tanhf(acc)) : 1.f;
}

// ---- backward ------------------------------------------------------------------------------
// dz = dL/dw * w * ln2 * (1 - tanh^2 z); dh = dz w_out
__global__ void k_sn_out_bwd(int64_t n, const float *__restrict__ z, const float *__restrict__ dw,
                             const float *__restrict__ p, float *__restrict__ dz, float *__restrict__ dh) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float th = tanhf(z[i]);
    const float d = dw[i] * expf(kOutC * th) * kOutC * (1.f - th * th);
    dz[i] = d;
#pragma unroll
    for (int k = 0; k < kSnW; ++k) dh[i * kSnW + k] = d * p[kSnOffWout + k];
}

// du = dh (u > 0); din = W^T du: dh += din[0:32] (the residual path and the h input), da = din[32:64]
__global__ void __launch_bounds__(128) k_sn_mlp_bwd(int64_t n, const float *__restrict__ W,
                                                    const float *__restrict__ u, float *__restrict__ dh,
                                                    float *__restrict__ du, float *__restrict__ da) {
    __shared__ float sw[kSnW * 2 * kSnW];
    for (int k = threadIdx.x; k < kSnW * 2 * kSnW; k += blockDim.x) sw[k] = W[k];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float d[kSnW];
#pragma unroll
    for (int o = 0; o < kSnW; ++o) {
        d[o] = u[i * kSnW + o] > 0.f ? dh[i * kSnW + o] : 0.f;
        du[i * kSnW + o] = d[o];
    }
    for (int k = 0; k < 2 * kSnW; ++k) {
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < kSnW; ++o) s += sw[o * 2 * kSnW + k] * d[o];
        if (k < kSnW) dh[i * kSnW + k] += s;
        else da[i * kSnW + k - kSnW] = s;
    }
}

// du0 = dh0 (u0 > 0), in place
__global__ void k_sn_relu_bwd(int64_t total, const float *__restrict__ u, float *__restrict__ d) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < total && !(u[t] > 0.f)) d[t] = 0.f;
}

// Weight gradient partials: block b sums over its rows [b*R, (b+1)*R) the outer product of
// du [n][O] with the input [in1 (K1 channels) ; in2 (K - K1 channels)], plus du itself (the
// bias): part[b][O*K + O].  Fixed rows per block and a fixed order: deterministic.
template <int O, int K, int K1>
__global__ void __launch_bounds__(256) k_sn_wgrad(int64_t n, int64_t rows_per_block, const float *__restrict__ du,
                                                  const float *__restrict__ in1, const float *__restrict__ in2,
                                                  float *__restrict__ part) {
    constexpr int E = O * K + O;
    constexpr int kTile = 32;
    __shared__ float sd[kTile][O];
    __shared__ float si[kTile][K];
    float acc[(E + 255) / 256];
#pragma unroll
    for (int q = 0; q < (E + 255) / 256; ++q) acc[q] = 0.f;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
    const int64_t r1 = min(n, r0 + rows_per_block);
    for (int64_t t0 = r0; t0 < r1; t0 += kTile) {
        __syncthreads();
        for (int e = threadIdx.x; e < kTile * O; e += blockDim.x) {
            const int64_t r = t0 + e / O;
            sd[e / O][e % O] = r < r1 ? du[r * O + e % O] : 0.f;
        }
        for (int e = threadIdx.x; e < kTile * K; e += blockDim.x) {
            const int64_t r = t0 + e / K;
            const int k = e % K;
            float v = 0.f;
            if (r < r1) v = k < K1 ? in1[r * K1 + k] : in2[r * (K - K1) + k - K1];
            si[e / K][k] = v;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < (E + 255) / 256; ++q) {
            const int e = q * 256 + threadIdx.x;
            if (e >= E) continue;
            float s = 0.f;
            if (e < O * K) {
                const int o = e / K, k = e % K;
                for (int rr = 0; rr < kTile; ++rr) s += sd[rr][o] * si[rr][k];
            } else {
                const int o = e - O * K;
                for (int rr = 0; rr < kTile; ++rr) s += sd[rr][o];
            }
            acc[q] += s;
        }
    }
#pragma unroll
    for (int q = 0; q < (E + 255) / 256; ++q) {
        const int e = q * 256 + threadIdx.x;
        if (e < E) part[(int64_t)blockIdx.x * E + e] = acc[q];
    }
}

// grad[dst + e] = sum over blocks of part[b][e] in block order (weights first, then biases,
// written to their places in the parameter vector)
__global__ void k_sn_wsum(int nb, int E, int OK, const float *__restrict__ part, float *__restrict__ grad, int w_off,
                          int b_off) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(int64_t)b * E + e];
    if (e < OK) grad[w_off + e] = (float)s;
    else grad[b_off + e - OK] = (float)s;
}

__global__ void k_sn_adam(int n, float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                          const float *__restrict__ g, float lr, float b1t, float b2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m[i] = 0.9f * m[i] + 0.1f * gi;
    v[i] = 0.999f * v[i] + 0.001f * gi * gi;
    const float mh = m[i] / (1.f - b1t), vh = v[i] / (1.f - b2t);
    w[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// ---- the cycle's adjoint pieces -------------------------------------------------------------
// y = S^ (w v) (w null: S^ v) over the solver rows
__global__ void k_sn_spmv(int64_t n, Sell A, const float *__restrict__ w, const float *__restrict__ v,
                          float *__restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t base;
    int wd, ln;
    sell_row(A, i, base, wd, ln);
    float acc = 0.f;
    for (int j = 0; j < wd; ++j) {
        const int64_t slot = base + (int64_t)j * kSliceRows + ln;
        const int32_t c = A.col[slot];
        acc += A.val[slot] * (w ? w[c] * v[c] : v[c]);
    }
    y[i] = acc;
}

// out = a + alpha * b
__global__ void k_sn_axpy(int64_t n, const float *__restrict__ a, float alpha, const float *__restrict__ b,
                          float *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] + alpha * b[i];
}

// per-block partial sums of x.y (fixed grid and order)
constexpr int kDotBlocks = 148;
__global__ void __launch_bounds__(256) k_sn_dot(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                                                double *__restrict__ part) {
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += (double)x[i] * y[i];
    __shared__ double sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sn_dot_total(const double *__restrict__ part, int nb, double *__restrict__ out) {
    if (threadIdx.x || blockIdx.x) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[b];
    *out = s;
}

// dL/dw_i = a0 (g_i r2_i + h_i r_i) + a1 (g_i (S^W r2)_i + (S^W g)_i r2_i + h_i (S^W r)_i
//           + (S^W h)_i r_i), zero on rows outside the hierarchy and padding rows; accumulated
__global__ void k_sn_grad_w(int64_t n, float a0, float a1, const float *__restrict__ g, const float *__restrict__ hh,
                            const float *__restrict__ r, const float *__restrict__ r2, const float *__restrict__ swr,
                            const float *__restrict__ swr2, const float *__restrict__ swg,
                            const float *__restrict__ swh, const int32_t *__restrict__ agg,
                            const int32_t *__restrict__ row_edge, float scale, float *__restrict__ dw) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (row_edge[i] < 0 || (agg && agg[i] < 0)) return;
    const float v = a0 * (g[i] * r2[i] + hh[i] * r[i]) +
                    a1 * (g[i] * swr2[i] + swg[i] * r2[i] + hh[i] * swr[i] + swh[i] * r[i]);
    dw[i] += scale * v;
}

inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

Sell sell_of(const DevSystem &s) { return {s.slice_off, s.col, s.val32}; }

}  // namespace

cudaError_t sn_features(const DevSystem &sys, float *x, cudaStream_t s) {
    k_sn_features<<<blocks(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sell_of(sys), sys.row_edge, x);
    return cudaGetLastError();
}

cudaError_t sn_forward(const DevSystem &sys, const float *params, const float *x, SnActs &act, float *w,
                       bool keep, cudaStream_t s) {
    const int64_t n = sys.n_rows;
    const Sell A = sell_of(sys);
    k_sn_layer0<<<blocks(n, 128), 128, 0, s>>>(n, x, params, keep ? act.u0 : nullptr, act.h[0]);
    for (int l = 0; l < kSnL; ++l) {
        k_sn_aggregate<false><<<blocks(n, 8), 256, 0, s>>>(n, A, act.h[keep ? l : (l & 1)], act.a[keep ? l : 0]);
        const float *W = params + kSnOffLayer + l * kSnPerLayer;
        float *hin = act.h[keep ? l : (l & 1)], *hout = act.h[keep ? l + 1 : ((l + 1) & 1)];
        k_sn_mlp<<<blocks(n, 128), 256, 0, s>>>(n, hin, act.a[keep ? l : 0], W, W + kSnW * 2 * kSnW,
                                                keep ? act.u[l] : nullptr, hout);
    }
    k_sn_out<<<blocks(n, 8), 256, 0, s>>>(n, act.h[keep ? kSnL : (kSnL & 1)], params, sys.row_edge,
                                         keep ? act.z : nullptr, w);
    return cudaGetLastError();
}

cudaError_t sn_backward(const DevSystem &sys, const float *params, const float *x, SnActs &act, const float *dw,
                        float *grad, SnScratch &sc, cudaStream_t s) {
    const int64_t n = sys.n_rows;
    const Sell A = sell_of(sys);
    const int64_t rpb = (n + kSnWgradBlocks - 1) / kSnWgradBlocks;
    const int nb = (int)((n + rpb - 1) / rpb);
    // output layer
    k_sn_out_bwd<<<blocks(n, 256), 256, 0, s>>>(n, act.z, dw, params, sc.dz, sc.dh);
    k_sn_wgrad<1, kSnW, kSnW><<<nb, 256, 0, s>>>(n, rpb, sc.dz, act.h[kSnL], nullptr, sc.part);
    k_sn_wsum<<<1, 64, 0, s>>>(nb, kSnW + 1, kSnW, sc.part, grad, kSnOffWout, kSnOffBout);
    for (int l = kSnL - 1; l >= 0; --l) {
        const float *W = params + kSnOffLayer + l * kSnPerLayer;
        k_sn_mlp_bwd<<<blocks(n, 128), 128, 0, s>>>(n, W, act.u[l], sc.dh, sc.du, sc.da);
        k_sn_wgrad<kSnW, 2 * kSnW, kSnW><<<nb, 256, 0, s>>>(n, rpb, sc.du, act.h[l], act.a[l], sc.part);
        const int E = kSnW * 2 * kSnW + kSnW;
        k_sn_wsum<<<blocks(E, 256), 256, 0, s>>>(nb, E, kSnW * 2 * kSnW, sc.part, grad, kSnOffLayer + l * kSnPerLayer,
                                                 kSnOffLayer + l * kSnPerLayer + kSnW * 2 * kSnW);
        // the message passing: dh += A^T da (A symmetric)
        k_sn_aggregate<true><<<blocks(n, 8), 256, 0, s>>>(n, A, sc.da, sc.dh);
    }
    k_sn_relu_bwd<<<blocks(n * kSnW, 256), 256, 0, s>>>(n * kSnW, act.u0, sc.dh);
    k_sn_wgrad<kSnW, kSnF, kSnF><<<nb, 256, 0, s>>>(n, rpb, sc.dh, x, nullptr, sc.part);
    const int E0 = kSnW * kSnF + kSnW;
    k_sn_wsum<<<blocks(E0, 256), 256, 0, s>>>(nb, E0, kSnW * kSnF, sc.part, grad, kSnOffW0, kSnOffB0);
    return cudaGetLastError();
}

cudaError_t sn_adam(float *params, float *m, float *v, const float *grad, int step, float lr, cudaStream_t s) {
    const float b1t = powf(0.9f, (float)step), b2t = powf(0.999f, (float)step);
    k_sn_adam<<<blocks(kSnParams, 256), 256, 0, s>>>(kSnParams, params, m, v, grad, lr, b1t, b2t);
    return cudaGetLastError();
}

cudaError_t sn_spmv(const DevSystem &sys, const float *w, const float *v, float *y, cudaStream_t s) {
    k_sn_spmv<<<blocks(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sell_of(sys), w, v, y);
    return cudaGetLastError();
}

cudaError_t sn_axpy(int64_t n, const float *a, float alpha, const float *b, float *out, cudaStream_t s) {
    k_sn_axpy<<<blocks(n, 256), 256, 0, s>>>(n, a, alpha, b, out);
    return cudaGetLastError();
}

cudaError_t sn_dot(int64_t n, const float *x, const float *y, double *part, double *out, cudaStream_t s) {
    k_sn_dot<<<kDotBlocks, 256, 0, s>>>(n, x, y, part);
    k_sn_dot_total<<<1, 32, 0, s>>>(part, kDotBlocks, out);
    return cudaGetLastError();
}

cudaError_t sn_grad_w(const DevSystem &sys, float a0, float a1, const float *g, const float *h, const float *r,
                      const float *r2, const float *swr, const float *swr2, const float *swg, const float *swh,
                      const int32_t *agg, float scale, float *dw, cudaStream_t s) {
    k_sn_grad_w<<<blocks(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, a0, a1, g, h, r, r2, swr, swr2, swg, swh, agg,
                                                       sys.row_edge, scale, dw);
    return cudaGetLastError();
}

}  // namespace mh
