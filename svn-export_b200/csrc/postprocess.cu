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

}  // namespace

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
