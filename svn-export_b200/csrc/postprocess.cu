// Flow post-processing on the device: the Darcy flux vector at every element centre from the
// side fluxes of the MH solution, DarcyFlowMHOutput::make_element_vector
// (src/flow/darcy_flow_mh_output.cc:301-323).  For each element E with sides s and side
// fluxes q_s, at the centre c (the mean of the nodes):
//     u_E = sum_s q_s RT0_s(c) / delta_E                          (delta_E: cross-section)
// with the lowest-order Raviart-Thomas basis of MHFEValues::RT0_value
// (src/flow/mh_fe_values.cc:76-118) and its parameters from the local-matrix routines:
//   line         RT0_0 = -|c - X_1| v / |v|^2,  RT0_1 = |c - X_0| v / |v|^2,  v = X_1 - X_0
//   triangle     RT0_s = g_s ((u.e_x - a_s) e_x + (u.e_y - b_s) e_y),  u = c - X_0, in the
//                element's plane frame (e_x along X_1 - X_0); (a_s, b_s) the node opposite
//                side s in that frame, g_s = 1 / (2 |E|) computed from the node coordinates
//                as bas_func_0_triangle does (:293-301)
//   tetrahedron  RT0_s = d_s (c - X_s),  X_s the node opposite side s,
//                d_s = 1 / (|S_s| n_s.(c_s - X_s))  (basis_functions_tetrahedron, :379-396)
// One thread per element, per-dimension element lists (no divergence between shapes); the
// output is [n_el][3], the three flux columns of the reference's raw output.
// Bytes per element: DIM+1 node indices and their coordinates (gathered, mostly from L2),
// DIM+1 side fluxes and the cross-section read, 24 bytes written.
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
    c = v3div(c, (double)N);
    const double cs = d.cross_section[e];
    const int s0 = d.el_side_start[e];
    V3 u = {0.0, 0.0, 0.0};
    auto add = [&](double q, V3 v) {  // u += q RT0_s(c) / delta, component by component
        u.x += q * v.x / cs;
        u.y += q * v.y / cs;
        u.z += q * v.z / cs;
    };
    if constexpr (DIM == 1) {
        const V3 v = v3sub(X[1], X[0]);
        const double ll = v3dot(v, v);
        add(sol[s0], v3scale(v, -v3norm(v3sub(c, X[1])) / ll));
        add(sol[s0 + 1], v3scale(v, v3norm(v3sub(c, X[0])) / ll));
    } else if constexpr (DIM == 2) {
        V3 ex = v3sub(X[1], X[0]);
        ex = v3div(ex, v3norm(ex));
        V3 ez = v3cross(ex, v3sub(X[2], X[0]));
        ez = v3div(ez, v3norm(ez));
        V3 ey = v3cross(ez, ex);
        ey = v3div(ey, v3norm(ey));
        double px[3], py[3];  // node coordinates in the plane frame
        px[0] = py[0] = 0.0;
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            const V3 dk = v3sub(X[k], X[0]);
            px[k] = v3dot(dk, ex);
            py[k] = v3dot(dk, ey);
        }
        const V3 w = v3sub(c, X[0]);
        const double wx = v3dot(w, ex), wy = v3dot(w, ey);
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int i0 = s, i1 = (s + 1) % 3, i2 = (s + 2) % 3;
            const double g = 1.0 / fabs((px[i0] - px[i2]) * (py[i1] - py[i0]) + (py[i0] - py[i2]) * (px[i0] - px[i1]));
            const double a = wx - px[i2], b = wy - py[i2];
            add(sol[s0 + s], {g * (a * ex.x + b * ey.x), g * (a * ex.y + b * ey.y), g * (a * ex.z + b * ey.z)});
        }
    } else {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const V3 a = X[dev_side_node(3, s, 0)], b = X[dev_side_node(3, s, 1)], q = X[dev_side_node(3, s, 2)];
            const V3 cr = v3cross(v3sub(b, a), v3sub(q, a));
            const double nr = v3norm(cr);
            V3 nv = v3div(cr, nr);
            if (v3dot(nv, v3sub(c, a)) > 0.0) nv = v3scale(nv, -1.0);  // outward
            const V3 sc = {(a.x + b.x + q.x) / 3.0, (a.y + b.y + q.y) / 3.0, (a.z + b.z + q.z) / 3.0};
            const double ds = 1.0 / (0.5 * nr * (v3dot(nv, sc) - v3dot(nv, X[s])));
            add(sol[s0 + s], v3scale(v3sub(c, X[s]), ds));
        }
    }
    out[3 * (int64_t)e] = u.x;
    out[3 * (int64_t)e + 1] = u.y;
    out[3 * (int64_t)e + 2] = u.z;
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
