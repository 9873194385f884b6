// Flow post-processing on the device: the Darcy flux vector at every element centre from the
// side fluxes of the MH solution, DarcyFlowMHOutput::make_element_vector
// (src/flow/darcy_flow_mh_output.cc:301-323).  For each element E with sides s and side
// fluxes q_s, at the centre c (the mean of the nodes):
//     u_E = sum_s q_s RT0_s(c) / delta_E                          (delta_E: cross-section)
// with the lowest-order Raviart-Thomas basis of MHFEValues::RT0_value
// (src/flow/mh_fe_values.cc:76-118).  The reference evaluates the basis from its local-matrix
// parameters (line :150-152, triangle :193-211 with bas_func_0_triangle :293-301, tetrahedron
// :379-396); at the centre each of those equals
//     RT0_s(c) = (c - X_opp(s)) / (dim |E|)
// with X_opp(s) the node opposite side s (line: the other node; triangle: node (s+2) mod 3;
// tetrahedron: node s): |S_s| times the height of X_s over side s is dim |E|, the triangle
// formula is that vector written in the element's plane frame, and the line's is
// -(|v|/2) v / |v|^2 = (c - X_1) / |v| for side 0.  So
//     u_E = sum_s q_s (c - X_opp(s)) / (dim |E| delta_E),
// one division per element instead of the reference's per-side normals, square roots and
// divisions (which made the literal version FP64-divide bound: 172 us for 1.57M tetrahedra).
// The oracle (oracle/mh_oracle.c, orc_element_flux) keeps the reference's literal formulas,
// so the parity tests also check the identity.
// One thread per element, per-dimension element lists (no divergence between shapes); the
// output is [n_el][3], the three flux columns of the reference's raw output.
// Bytes per element: DIM+1 node indices and their coordinates (gathered, mostly from L2),
// DIM+1 side fluxes, the side offset, the cross-section and the list entry read, 24 written.
#include <cuda_runtime.h>

#include "device_system.hpp"
#include "mh_local.cuh"

namespace mh {
namespace {

template <int DIM>
__global__ void __launch_bounds__(128) k_element_flux(ElemData d, const int32_t *__restrict__ list, int64_t n,
                                                      const double *__restrict__ sol, double *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int e = list[t];
    constexpr int N = DIM + 1;
    V3 X[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const int nd = d.el_nodes[4 * e + i];
        X[i] = {d.xyz[3 * nd], d.xyz[3 * nd + 1], d.xyz[3 * nd + 2]};
    }
    V3 c = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < N; ++i) c = {c.x + X[i].x, c.y + X[i].y, c.z + X[i].z};
    c = v3scale(c, 1.0 / N);
    double dm;  // dim |E|
    if constexpr (DIM == 1) {
        dm = v3norm(v3sub(X[1], X[0]));
    } else if constexpr (DIM == 2) {
        dm = v3norm(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0])));
    } else {
        dm = fabs(v3dot(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0])), v3sub(X[3], X[0]))) / 2.0;
    }
    const double f = 1.0 / (dm * d.cross_section[e]);
    const int s0 = d.el_side_start[e];
    V3 u = {0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < N; ++s) {
        const int opp = DIM == 1 ? 1 - s : DIM == 2 ? (s + 2) % 3 : s;
        const double q = sol[s0 + s];
        const V3 r = v3sub(c, X[opp]);
        u = {u.x + q * r.x, u.y + q * r.y, u.z + q * r.z};
    }
    out[3 * (int64_t)e] = u.x * f;
    out[3 * (int64_t)e + 1] = u.y * f;
    out[3 * (int64_t)e + 2] = u.z * f;
}

// ---- node pressures (make_node_scalar_param, darcy_flow_mh_output.cc:424-546) ---------------
// A node's pressure is the mean of the pressures of the elements and element sides that
// contain it, weighted by (1 - d / D) / (n - 1): d the distance from the node to that element's
// or side's centre, D the sum of those distances at the node, n their number.  Pass 1 adds
// the distances and counts, pass 2 the weighted pressures, both by FP64 atomics into per-node
// sums (the summation order varies between runs in the last bits).
template <int DIM, int PASS>
__global__ void __launch_bounds__(128) k_node_pressure(ElemData d, const int32_t *__restrict__ list, int64_t n,
                                                       const double *__restrict__ sol, int64_t n_sides, int64_t n_el,
                                                       double *__restrict__ dsum, int32_t *__restrict__ cnt,
                                                       double *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int e = list[t];
    constexpr int N = DIM + 1;
    V3 X[N];
    int nd[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        nd[i] = d.el_nodes[4 * e + i];
        X[i] = {d.xyz[3 * nd[i]], d.xyz[3 * nd[i] + 1], d.xyz[3 * nd[i] + 2]};
    }
    auto visit = [&](int k, V3 centre, double p) {
        const double dist = v3norm(v3sub(X[k], centre));
        if (PASS == 0) {
            atomicAdd(dsum + nd[k], dist);
            atomicAdd(cnt + nd[k], 1);
        } else {
            atomicAdd(out + nd[k], p * (1.0 - dist / dsum[nd[k]]) / (cnt[nd[k]] - 1));
        }
    };
    V3 c = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < N; ++i) c = {c.x + X[i].x, c.y + X[i].y, c.z + X[i].z};
    c = v3div(c, (double)N);
    const double pe = PASS ? sol[n_sides + e] : 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) visit(k, c, pe);
    const int s0 = d.el_side_start[e];
#pragma unroll
    for (int s = 0; s < N; ++s) {  // side s has DIM nodes
        V3 cs = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            const V3 q = X[dev_side_node(DIM, s, k)];
            cs = {cs.x + q.x, cs.y + q.y, cs.z + q.z};
        }
        cs = v3div(cs, (double)DIM);
        const double ps = PASS ? sol[n_sides + n_el + d.side_edge[s0 + s]] : 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) visit(dev_side_node(DIM, s, k), cs, ps);
    }
}

// ---- water balance (water_balance, darcy_flow_mh_output.cc:671-790) ----------------------------
// Per boundary region the sum of the outward side fluxes of its boundary objects, of the positive
// ones and of the negative ones; per bulk region the sum of |E| delta_E f_E.  Each block adds into
// shared per-region partials and then once per region into the global sums (FP64 atomics).
constexpr int kBalanceSharedRegions = 512;

__global__ void __launch_bounds__(256) k_boundary_balance(ElemData d, int64_t n_sides, const double *__restrict__ sol,
                                                          const int32_t *__restrict__ bdr_region, int32_t n_reg,
                                                          double *__restrict__ out) {
    __shared__ double acc[3 * kBalanceSharedRegions];
    const bool shared = n_reg <= kBalanceSharedRegions;
    if (shared)
        for (int r = threadIdx.x; r < 3 * n_reg; r += blockDim.x) acc[r] = 0.0;
    __syncthreads();
    double *dst = shared ? acc : out;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_sides; s += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = d.side_bdr[s];
        if (b < 0) continue;
        const int32_t r = bdr_region[b];
        const double q = sol[s];
        atomicAdd(dst + 3 * r, q);
        atomicAdd(dst + 3 * r + (q > 0.0 ? 1 : 2), q);
    }
    __syncthreads();
    if (shared)
        for (int r = threadIdx.x; r < 3 * n_reg; r += blockDim.x)
            if (acc[r] != 0.0) atomicAdd(out + r, acc[r]);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_source_balance(ElemData d, const int32_t *__restrict__ list, int64_t n,
                                                        const int32_t *__restrict__ el_region, int32_t n_reg,
                                                        double *__restrict__ out) {
    __shared__ double acc[kBalanceSharedRegions];
    const bool shared = n_reg <= kBalanceSharedRegions;
    if (shared)
        for (int r = threadIdx.x; r < n_reg; r += blockDim.x) acc[r] = 0.0;
    __syncthreads();
    double *dst = shared ? acc : out;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int e = list[t];
        const double f = d.source[e];
        if (f == 0.0) continue;
        V3 X[DIM + 1];
#pragma unroll
        for (int i = 0; i <= DIM; ++i) {
            const int nd = d.el_nodes[4 * e + i];
            X[i] = {d.xyz[3 * nd], d.xyz[3 * nd + 1], d.xyz[3 * nd + 2]};
        }
        double meas;
        if constexpr (DIM == 1) {
            meas = v3norm(v3sub(X[1], X[0]));
        } else if constexpr (DIM == 2) {
            meas = v3norm(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0]))) / 2.0;
        } else {
            meas = fabs(v3dot(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0])), v3sub(X[3], X[0]))) / 6.0;
        }
        atomicAdd(dst + el_region[e], meas * d.cross_section[e] * f);
    }
    __syncthreads();
    if (shared)
        for (int r = threadIdx.x; r < n_reg; r += blockDim.x)
            if (acc[r] != 0.0) atomicAdd(out + r, acc[r]);
}

}  // namespace

cudaError_t launch_node_pressure(const ElemData &d, const DevAssembly &a, const double *sol, int64_t n_nodes,
                                 int64_t n_sides, int64_t n_el, double *dsum, int32_t *cnt, double *out,
                                 cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(dsum, 0, n_nodes * sizeof(double), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(cnt, 0, n_nodes * sizeof(int32_t), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(out, 0, n_nodes * sizeof(double), s)) != cudaSuccess) return e;
    auto blocks = [](int64_t n) { return (unsigned)((n + 127) / 128); };
#define MH_NODE_PASS(P)                                                                                        \
    if (a.dim_count[1] > 0)                                                                                    \
        k_node_pressure<1, P><<<blocks(a.dim_count[1]), 128, 0, s>>>(d, a.dim_list[1], a.dim_count[1], sol, n_sides, \
                                                                     n_el, dsum, cnt, out);                    \
    if (a.dim_count[2] > 0)                                                                                    \
        k_node_pressure<2, P><<<blocks(a.dim_count[2]), 128, 0, s>>>(d, a.dim_list[2], a.dim_count[2], sol, n_sides, \
                                                                     n_el, dsum, cnt, out);                    \
    if (a.dim_count[3] > 0)                                                                                    \
        k_node_pressure<3, P><<<blocks(a.dim_count[3]), 128, 0, s>>>(d, a.dim_list[3], a.dim_count[3], sol, n_sides, \
                                                                     n_el, dsum, cnt, out);
    MH_NODE_PASS(0)
    MH_NODE_PASS(1)
#undef MH_NODE_PASS
    return cudaGetLastError();
}

cudaError_t launch_water_balance(const ElemData &d, const DevAssembly &a, const double *sol, int64_t n_sides,
                                 const int32_t *bdr_region, int32_t n_bdr_reg, const int32_t *el_region,
                                 int32_t n_el_reg, double *bdr_out, double *src_out, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(bdr_out, 0, 3 * (size_t)n_bdr_reg * sizeof(double), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(src_out, 0, (size_t)n_el_reg * sizeof(double), s)) != cudaSuccess) return e;
    if (n_sides > 0)
        k_boundary_balance<<<296, 256, 0, s>>>(d, n_sides, sol, bdr_region, n_bdr_reg, bdr_out);
    if (a.dim_count[1] > 0)
        k_source_balance<1><<<148, 256, 0, s>>>(d, a.dim_list[1], a.dim_count[1], el_region, n_el_reg, src_out);
    if (a.dim_count[2] > 0)
        k_source_balance<2><<<148, 256, 0, s>>>(d, a.dim_list[2], a.dim_count[2], el_region, n_el_reg, src_out);
    if (a.dim_count[3] > 0)
        k_source_balance<3><<<296, 256, 0, s>>>(d, a.dim_list[3], a.dim_count[3], el_region, n_el_reg, src_out);
    return cudaGetLastError();
}

cudaError_t launch_element_flux(const ElemData &d, const DevAssembly &a, const double *sol, double *out,
                                cudaStream_t s) {
    auto blocks = [](int64_t n) { return (unsigned)((n + 127) / 128); };
    if (a.dim_count[1] > 0)
        k_element_flux<1><<<blocks(a.dim_count[1]), 128, 0, s>>>(d, a.dim_list[1], a.dim_count[1], sol, out);
    if (a.dim_count[2] > 0)
        k_element_flux<2><<<blocks(a.dim_count[2]), 128, 0, s>>>(d, a.dim_list[2], a.dim_count[2], sol, out);
    if (a.dim_count[3] > 0)
        k_element_flux<3><<<blocks(a.dim_count[3]), 128, 0, s>>>(d, a.dim_list[3], a.dim_count[3], sol, out);
    return cudaGetLastError();
}

}  // namespace mh
