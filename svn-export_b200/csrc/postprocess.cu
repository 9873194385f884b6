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
// or side's centre, D the sum of those distances at the node, n their number.  One thread per
// node gathers over the node's elements (ascending, from a CSR incidence list built once per
// mesh): first every element centre, then every side of those elements that contains the node,
// the order in which the reference's two element loops reach the node.  No atomics: repeated
// calls give identical bits, and with the operation order of the reference (this file is
// compiled without FMA contraction) the result equals the FP64 restatement bit for bit.
__device__ __forceinline__ double node_dist(V3 a, V3 b) {
    const V3 d = v3sub(a, b);
    return sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
}

__global__ void __launch_bounds__(128) k_node_pressure(ElemData d, const int32_t *__restrict__ inc_start,
                                                       const int32_t *__restrict__ inc_el, int64_t n_nodes,
                                                       const double *__restrict__ sol, int64_t n_sides, int64_t n_el,
                                                       double *__restrict__ out) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_nodes) return;
    const V3 Xv = {d.xyz[3 * v], d.xyz[3 * v + 1], d.xyz[3 * v + 2]};
    const int32_t p0 = inc_start[v], p1 = inc_start[v + 1];
    double D = 0.0, acc = 0.0;
    int cnt = 0;
    // pass 0: distance sum and count; pass 1: weighted pressures (same visiting order)
    for (int pass = 0; pass < 2; ++pass) {
        for (int32_t q = p0; q < p1; ++q) {  // element centres
            const int e = inc_el[q];
            const int N = d.el_side_start[e + 1] - d.el_side_start[e];
            V3 c = {0.0, 0.0, 0.0};
            for (int i = 0; i < N; ++i) {
                const int nd = d.el_nodes[4 * e + i];
                c = {c.x + d.xyz[3 * nd], c.y + d.xyz[3 * nd + 1], c.z + d.xyz[3 * nd + 2]};
            }
            c = v3div(c, (double)N);
            const double dist = node_dist(Xv, c);
            if (pass == 0) {
                D += dist;
                ++cnt;
            } else {
                acc += sol[n_sides + e] * (1.0 - dist / D) / (cnt - 1);
            }
        }
        for (int32_t q = p0; q < p1; ++q) {  // sides containing the node
            const int e = inc_el[q];
            const int s0 = d.el_side_start[e];
            const int N = d.el_side_start[e + 1] - s0, dim = N - 1;
            int nd[4];
            int kv = 0;
            for (int i = 0; i < N; ++i) {
                nd[i] = d.el_nodes[4 * e + i];
                if (nd[i] == v) kv = i;
            }
            for (int s = 0; s < N; ++s) {
                bool has = false;
                for (int k = 0; k < dim; ++k) has |= dev_side_node(dim, s, k) == kv;
                if (!has) continue;
                V3 cs = {0.0, 0.0, 0.0};
                for (int k = 0; k < dim; ++k) {
                    const int m = nd[dev_side_node(dim, s, k)];
                    cs = {cs.x + d.xyz[3 * m], cs.y + d.xyz[3 * m + 1], cs.z + d.xyz[3 * m + 2]};
                }
                cs = v3div(cs, (double)dim);
                const double dist = node_dist(Xv, cs);
                if (pass == 0) {
                    D += dist;
                    ++cnt;
                } else {
                    acc += sol[n_sides + n_el + d.side_edge[s0 + s]] * (1.0 - dist / D) / (cnt - 1);
                }
            }
        }
    }
    out[v] = acc;
}

// ---- water balance (water_balance, darcy_flow_mh_output.cc:671-790) ----------------------------
// Per boundary region the sum of the outward side fluxes of its boundary objects, of the positive
// ones and of the negative ones; per bulk region the sum of |E| delta_E f_E.  The items (boundary
// sides, elements) come grouped by region in ascending order, cut into fixed chunks of at most
// kBalanceChunkItems items (host-built); one block per chunk sums it in a fixed order (strided
// per-thread sums, then a fixed tree), and one thread per region adds its chunks in order:
// deterministic, no atomics.

template <int NV> __device__ __forceinline__ void block_tree(double (&v)[NV], double (*sh)[NV]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[t][k] = v[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w)
#pragma unroll
            for (int k = 0; k < NV; ++k) sh[t][k] += sh[t + w][k];
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = sh[0][k];
}

// KIND 0: boundary sides (total, outflow, inflow); KIND 1: element sources
template <int KIND>
__global__ void __launch_bounds__(256) k_balance_chunks(ElemData d, const double *__restrict__ sol,
                                                        const int32_t *__restrict__ items,
                                                        const int64_t *__restrict__ chunk_begin,
                                                        double *__restrict__ partial) {
    constexpr int NV = KIND == 0 ? 3 : 1;
    __shared__ double sh[256][NV];
    const int64_t b0 = chunk_begin[blockIdx.x], b1 = chunk_begin[blockIdx.x + 1];
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int64_t t = b0 + threadIdx.x; t < b1; t += blockDim.x) {
        const int32_t it = items[t];
        if constexpr (KIND == 0) {
            const double q = sol[it];
            v[0] += q;
            if (q > 0.0) v[1] += q;
            else v[2] += q;
        } else {
            const int e = it;
            const double f = d.source[e];
            if (f == 0.0) continue;
            const int N = d.el_side_start[e + 1] - d.el_side_start[e];
            V3 X[4];
            for (int i = 0; i < N; ++i) {
                const int nd = d.el_nodes[4 * e + i];
                X[i] = {d.xyz[3 * nd], d.xyz[3 * nd + 1], d.xyz[3 * nd + 2]};
            }
            double meas;
            if (N == 2) {
                meas = v3norm(v3sub(X[1], X[0]));
            } else if (N == 3) {
                meas = v3norm(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0]))) / 2.0;
            } else {
                meas = fabs(v3dot(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0])), v3sub(X[3], X[0]))) / 6.0;
            }
            v[0] += meas * d.cross_section[e] * f;
        }
    }
    block_tree<NV>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) partial[(int64_t)blockIdx.x * NV + k] = v[k];
}

template <int NV>
__global__ void k_balance_regions(const int64_t *__restrict__ region_chunk, int32_t n_reg,
                                  const double *__restrict__ partial, double *__restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reg) return;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int64_t c = region_chunk[r]; c < region_chunk[r + 1]; ++c)
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += partial[c * NV + k];
#pragma unroll
    for (int k = 0; k < NV; ++k) out[(int64_t)r * NV + k] = v[k];
}

}  // namespace

cudaError_t launch_node_pressure(const ElemData &d, const int32_t *inc_start, const int32_t *inc_el, int64_t n_nodes,
                                 const double *sol, int64_t n_sides, int64_t n_el, double *out, cudaStream_t s) {
    if (n_nodes > 0)
        k_node_pressure<<<(unsigned)((n_nodes + 127) / 128), 128, 0, s>>>(d, inc_start, inc_el, n_nodes, sol, n_sides,
                                                                          n_el, out);
    return cudaGetLastError();
}

cudaError_t launch_water_balance(const ElemData &d, const double *sol, const BalanceLists &L, double *partial,
                                 double *bdr_out, double *src_out, cudaStream_t s) {
    if (L.n_bdr_chunks > 0)
        k_balance_chunks<0><<<(unsigned)L.n_bdr_chunks, 256, 0, s>>>(d, sol, L.bdr_items, L.bdr_chunk_begin, partial);
    k_balance_regions<3><<<(unsigned)((L.n_bdr_reg + 127) / 128), 128, 0, s>>>(L.bdr_region_chunk, L.n_bdr_reg, partial,
                                                                               bdr_out);
    double *sp = partial + 3 * L.n_bdr_chunks;
    if (L.n_src_chunks > 0)
        k_balance_chunks<1><<<(unsigned)L.n_src_chunks, 256, 0, s>>>(d, sol, L.src_items, L.src_chunk_begin, sp);
    k_balance_regions<1><<<(unsigned)((L.n_src_reg + 127) / 128), 128, 0, s>>>(L.src_region_chunk, L.n_src_reg, sp,
                                                                               src_out);
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
