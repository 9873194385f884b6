// K1 (local MH + double Schur elimination, scattered into SELL-C-sigma), the diagonal
// scaling, and K4 (back-substitution of element pressures and side fluxes).
//
// K1 replaces assembly_steady_mh_matrix (src/flow/darcy_flow_mh.cc:525-694), the IA1 refill
// of make_schur1 (:1062-1075), SchurComplement::form_schur/form_rhs (src/la/schur.cc:566-611,
// 690-694) and make_schur2 (darcy_flow_mh.cc:1095-1131).  Because B only couples an element
// to its own sides and the element diagonal of S1 is a scalar, both eliminations are local:
// one thread computes an element's whole (n+k)x(n+k) contribution to the edge system.
// The contributions are summed per SELL slot by a gather over a host-built contribution
// list (element order), so the result is deterministic and needs no atomics.
#include <cuda_runtime.h>

#include "device_system.hpp"
#include "mh_local.cuh"

namespace mh {

namespace {

constexpr int kModeMatrix = 1;
constexpr int kModeRhs = 2;

template <int DIM, int G>
__global__ void __launch_bounds__(G) k1_local_blocks(ElemData d, const int32_t *__restrict__ list, int64_t n,
                                                       const int64_t *__restrict__ blk_off,
                                                       const int64_t *__restrict__ rhs_off, double *__restrict__ blk,
                                                       double *__restrict__ rhs_loc, int mode, int32_t *status) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int e = list[t];
    LocalMH<DIM> L;
    build_local<DIM>(d, e, L);
    constexpr int N = DIM + 1;
    const int m = N + L.k;
    int bad = L.singular ? 1 : 0;
    if (mode & kModeMatrix) {
        double *B = blk + blk_off[e];
#pragma unroll
        for (int l = 0; l < LocalMH<DIM>::M; ++l) {
            if (l >= m) break;
#pragma unroll
            for (int c = 0; c < LocalMH<DIM>::M; ++c) {
                if (c >= m) break;
                double v = local_s2<DIM>(L, l, c);
                if (!isfinite(v)) bad |= 2;
                B[l * m + c] = v;
            }
        }
    }
    if (mode & kModeRhs) {
        double *rl = rhs_loc + rhs_off[e];
#pragma unroll
        for (int l = 0; l < LocalMH<DIM>::M; ++l) {
            if (l >= m) break;
            double v = local_r2<DIM>(L, l);
            if (!isfinite(v)) bad |= 2;
            rl[l] = v;
        }
    }
    if (bad) atomicOr(status, bad);
}

// One thread per solver row: sum the contributions of every slot of the row (matrix) and
// of the row's rhs entry.  Padding rows become identity rows with zero rhs.
__global__ void __launch_bounds__(256) k1_gather(int64_t n_rows, const int64_t *__restrict__ slice_off,
                                                 const int32_t *__restrict__ row_edge,
                                                 const int32_t *__restrict__ slot_cstart,
                                                 const int32_t *__restrict__ slot_cidx,
                                                 const double *__restrict__ blk,
                                                 const int32_t *__restrict__ row_cstart,
                                                 const int32_t *__restrict__ row_cidx,
                                                 const double *__restrict__ rhs_loc, double *__restrict__ val,
                                                 double *__restrict__ b, int mode) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    const bool pad = row_edge[row] < 0;
    if (mode & kModeMatrix) {
        const int64_t sl = row / kSliceRows;
        const int lane = (int)(row % kSliceRows);
        const int64_t off = slice_off[sl];
        const int w = (int)((slice_off[sl + 1] - off) / kSliceRows);
        for (int j = 0; j < w; ++j) {
            const int64_t slot = off + (int64_t)j * kSliceRows + lane;
            double s = 0.0;
            if (pad) {
                s = (j == 0) ? 1.0 : 0.0;
            } else {
                for (int k = slot_cstart[slot]; k < slot_cstart[slot + 1]; ++k) s += blk[slot_cidx[k]];
            }
            val[slot] = s;
        }
    }
    if (mode & kModeRhs) {
        double s = 0.0;
        if (!pad)
            for (int k = row_cstart[row]; k < row_cstart[row + 1]; ++k) s += rhs_loc[row_cidx[k]];
        b[row] = s;
    }
}

__global__ void k_scale_diag(int64_t n_rows, const int32_t *__restrict__ diag_slot, const double *__restrict__ val,
                             double *__restrict__ dsq) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    double dg = val[diag_slot[row]];
    dsq[row] = sqrt(dg > 0.0 ? dg : 1.0);
}

__global__ void __launch_bounds__(256) k_scale_values(int64_t n_rows, const int64_t *__restrict__ slice_off,
                                                      const int32_t *__restrict__ col, const double *__restrict__ val,
                                                      const double *__restrict__ dsq, double *__restrict__ v64,
                                                      float *__restrict__ v32) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    const int64_t sl = row / kSliceRows;
    const int lane = (int)(row % kSliceRows);
    const int64_t off = slice_off[sl];
    const int w = (int)((slice_off[sl + 1] - off) / kSliceRows);
    const double di = dsq[row];
    for (int j = 0; j < w; ++j) {
        const int64_t slot = off + (int64_t)j * kSliceRows + lane;
        const double v = val[slot] / (di * dsq[col[slot]]);
        v64[slot] = v;
        v32[slot] = (float)v;
    }
}

__global__ void k_scale_rhs(int64_t n_rows, const double *__restrict__ b, const double *__restrict__ dsq,
                            double *__restrict__ bh) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    bh[row] = b[row] / dsq[row];
}

// x[row] = lambda[edge(row)] * dsq[row]: an edge-pressure guess in scaled space.
__global__ void k_scale_in(int64_t n_rows, const int32_t *__restrict__ row_edge, const double *__restrict__ lambda,
                           const double *__restrict__ dsq, double *__restrict__ x) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    const int e = row_edge[row];
    x[row] = (e >= 0) ? lambda[e] * dsq[row] : 0.0;
}

// lambda[e] = x[row(e)] / dsq[row(e)], written into the edge part of the MH solution.
__global__ void k_unscale(int64_t n_edges, const int32_t *__restrict__ edge_row, const double *__restrict__ x,
                          const double *__restrict__ dsq, double *__restrict__ lambda) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    const int r = edge_row[e];
    lambda[e] = x[r] / dsq[r];
}

// K4: p_E = (r1_E - S1_Ef lambda) / S1_EE  (schur2 resolve, schur.cc:738-745)
//     q_E = A_E^-1 (g + p_E - c .* lambda_own) (schur1 resolve)
// plus, for LMH, the flux correction of DarcyFlowLMH_Unsteady::postprocess
// (darcy_flow_mh.cc:1772-1827).
template <int DIM>
__global__ void __launch_bounds__(128) k4_backsub(ElemData d, const int32_t *__restrict__ list, int64_t n,
                                                  const double *__restrict__ lambda, double *__restrict__ sol,
                                                  int64_t n_sides) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int e = list[t];
    LocalMH<DIM> L;
    build_local<DIM>(d, e, L);
    constexpr int N = DIM + 1;
    double acc = L.r1e;
#pragma unroll
    for (int l = 0; l < LocalMH<DIM>::M; ++l)
        if (l < N + L.k) acc -= L.u[l] * lambda[L.edge[l]];
    const double pE = acc / L.s1ee;
    double rhs[N];
#pragma unroll
    for (int i = 0; i < N; ++i) rhs[i] = L.g[i] + pE - L.c[i] * lambda[L.edge[i]];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double q = 0.0;
#pragma unroll
        for (int j = 0; j < N; ++j) q += L.Ainv[i][j] * rhs[j];
        if (d.time_mode == 2) q += -L.lmh_coef * (lambda[L.edge[i]] - d.prev_edge[L.edge[i]]) + L.src_side;
        sol[L.side0 + i] = q;
    }
    sol[n_sides + e] = pE;
}

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

template <int G>
void local_blocks_group(const ElemData &d, const DevAssembly &a, int mode, cudaStream_t s) {
    if (a.dim_count[1] > 0)
        k1_local_blocks<1, G><<<blocks_for(a.dim_count[1], G), G, 0, s>>>(
            d, a.dim_list[1], a.dim_count[1], a.blk_off, a.rhs_off, a.blk, a.rhs_loc, mode, a.status);
    if (a.dim_count[2] > 0)
        k1_local_blocks<2, G><<<blocks_for(a.dim_count[2], G), G, 0, s>>>(
            d, a.dim_list[2], a.dim_count[2], a.blk_off, a.rhs_off, a.blk, a.rhs_loc, mode, a.status);
    if (a.dim_count[3] > 0)
        k1_local_blocks<3, G><<<blocks_for(a.dim_count[3], G), G, 0, s>>>(
            d, a.dim_list[3], a.dim_count[3], a.blk_off, a.rhs_off, a.blk, a.rhs_loc, mode, a.status);
}

cudaError_t launch_local_blocks(const ElemData &d, const DevAssembly &a, int mode, int group, cudaStream_t s) {
    switch (group) {
        case 64: local_blocks_group<64>(d, a, mode, s); break;
        case 256: local_blocks_group<256>(d, a, mode, s); break;
        default: local_blocks_group<128>(d, a, mode, s); break;
    }
    return cudaGetLastError();
}

// constant additions (mortar coupling): one thread per slot, each slot once
__global__ void k_add_slots(int64_t n, const int32_t *__restrict__ slot, const double *__restrict__ v,
                            double *__restrict__ val) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) val[slot[k]] += v[k];
}

cudaError_t launch_gather(const DevAssembly &a, const DevSystem &sys, int mode, cudaStream_t s) {
    k1_gather<<<blocks_for(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sys.slice_off, sys.row_edge, a.slot_cstart,
                                                           a.slot_cidx, a.blk, a.row_cstart, a.row_cidx, a.rhs_loc,
                                                           sys.val_raw, sys.b, mode);
    if ((mode & 1) && a.n_add > 0)
        k_add_slots<<<blocks_for(a.n_add, 256), 256, 0, s>>>(a.n_add, a.add_slot, a.add_val, sys.val_raw);
    return cudaGetLastError();
}

cudaError_t launch_scale(const DevSystem &sys, int matrix, cudaStream_t s) {
    if (matrix) {
        k_scale_diag<<<blocks_for(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sys.diag_slot, sys.val_raw, sys.dsq);
        k_scale_values<<<blocks_for(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sys.slice_off, sys.col,
                                                                    sys.val_raw, sys.dsq, sys.val64, sys.val32);
    }
    k_scale_rhs<<<blocks_for(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sys.b, sys.dsq, sys.bh);
    return cudaGetLastError();
}

cudaError_t launch_scale_in(const DevSystem &sys, const double *lambda, cudaStream_t s) {
    k_scale_in<<<blocks_for(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sys.row_edge, lambda, sys.dsq, sys.x);
    return cudaGetLastError();
}

cudaError_t launch_backsub(const ElemData &d, const DevAssembly &a, const DevSystem &sys, double *sol,
                           int64_t n_sides, int64_t n_el, int64_t n_edges, cudaStream_t s) {
    double *lambda = sol + n_sides + n_el;
    k_unscale<<<blocks_for(n_edges, 256), 256, 0, s>>>(n_edges, sys.edge_row, sys.x, sys.dsq, lambda);
    if (a.dim_count[1] > 0)
        k4_backsub<1><<<blocks_for(a.dim_count[1], 128), 128, 0, s>>>(d, a.dim_list[1], a.dim_count[1], lambda, sol,
                                                                       n_sides);
    if (a.dim_count[2] > 0)
        k4_backsub<2><<<blocks_for(a.dim_count[2], 128), 128, 0, s>>>(d, a.dim_list[2], a.dim_count[2], lambda, sol,
                                                                       n_sides);
    if (a.dim_count[3] > 0)
        k4_backsub<3><<<blocks_for(a.dim_count[3], 128), 128, 0, s>>>(d, a.dim_list[3], a.dim_count[3], lambda, sol,
                                                                       n_sides);
    return cudaGetLastError();
}

}  // namespace mh
