// The convection matrix of Flow123d's explicit finite-volume transport from the side fluxes of
// the MH solution: ConvectionTransport::create_transport_matrix_mpi
// (src/transport/transport.cc:788-923), the consumer of the flow result.  Row i belongs to
// element i, V_i = |E_i| delta_i porosity_i, q the side fluxes (outward positive):
//   edge neighbour j (across a side of i not on a boundary object, through each other side s
//   of the same edge):   a_ij = -(q_i q_s / (Q_e |E_i| delta_i por_i)) if q_s > 0 and q_i < 0,
//                        else 0; Q_e = the sum of the positive side fluxes of the edge
//   VB, i the lower-dimensional element, q the flux of the higher element j's side:
//                        a_ij = q / V_i if q > 0, else 0
//   VB, i the higher-dimensional element of that side:  a_ij = -q / V_i if q < 0, else 0
//   diagonal             a_ii = -sum_{sides, q > 0} q / V_i - sum_{VB of i, q < 0} (-q) / V_i
// and cfl_max_step = 1 / max |a_ii|.  The sparsity pattern depends on the mesh only: the host
// builds it once per handle as "slots" (column, kind, side indices) sorted by column within each
// row, so the CSR column order is canonical; the values are recomputed on the device for every
// flux field, one thread per row, deterministically (the max is order-independent).  The
// arithmetic keeps the reference's operation order: divisions by ((|E| delta) por) and
// (((Q_e |E|) delta) por).
#include <cuda_runtime.h>

#include "device_system.hpp"
#include "mh_local.cuh"

namespace mh {
namespace {

__global__ void k_edge_outflow(int64_t n_edges, const int32_t *__restrict__ start, const int32_t *__restrict__ sides,
                               const double *__restrict__ sol, double *__restrict__ flow) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    double f = 0.0;
    for (int32_t k = start[e]; k < start[e + 1]; ++k) {
        const double q = sol[sides[k]];
        if (q > 0.0) f += q;
    }
    flow[e] = f;
}

__device__ __forceinline__ double element_measure(const ElemData &d, int e) {
    int nd[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) nd[i] = d.el_nodes[4 * e + i];
    auto P = [&](int i) { return V3{d.xyz[3 * nd[i]], d.xyz[3 * nd[i] + 1], d.xyz[3 * nd[i] + 2]}; };
    if (nd[2] < 0) return v3norm(v3sub(P(1), P(0)));
    if (nd[3] < 0) return v3norm(v3cross(v3sub(P(1), P(0)), v3sub(P(2), P(0)))) / 2.0;
    return fabs(v3dot(v3cross(v3sub(P(1), P(0)), v3sub(P(2), P(0))), v3sub(P(3), P(0)))) / 6.0;
}

__global__ void __launch_bounds__(128) k_transport_rows(ElemData d, int64_t n_el, const int32_t *__restrict__ row_ptr,
                                                        const int32_t *__restrict__ kind,
                                                        const int32_t *__restrict__ slot_a,
                                                        const int32_t *__restrict__ slot_b,
                                                        const int32_t *__restrict__ ngh_side,
                                                        const double *__restrict__ edge_flow,
                                                        const double *__restrict__ porosity,
                                                        const double *__restrict__ sol, double *__restrict__ val,
                                                        unsigned long long *__restrict__ diag_max) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double adiag = 0.0;
    if (i < n_el) {
        const double m = element_measure(d, (int)i), cs = d.cross_section[i];
        const double por = porosity ? porosity[i] : 1.0;
        const double v = (m * cs) * por;
        double aii = 0.0;
        for (int32_t s = d.el_side_start[i]; s < d.el_side_start[i + 1]; ++s) {
            const double q = sol[s];
            if (q > 0.0) aii -= q / v;
        }
        for (int32_t k = d.el_ngh_start[i]; k < d.el_ngh_start[i + 1]; ++k) {
            const double q = sol[ngh_side[d.el_ngh[k]]];
            if (q < 0.0) aii -= (-q) / v;
        }
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            double a = 0.0;
            switch (kind[k]) {
                case kTrDiag:
                    a = aii;
                    break;
                case kTrEdge: {
                    const double q = sol[slot_a[k]], q2 = sol[slot_b[k]];
                    if (q2 > 0.0 && q < 0.0) a = -(q * q2 / (((edge_flow[d.side_edge[slot_a[k]]] * m) * cs) * por));
                    break;
                }
                case kTrVbLower: {
                    const double q = sol[slot_a[k]];
                    if (q > 0.0) a = q / v;
                    break;
                }
                default: {  // kTrVbHigher
                    const double q = sol[slot_a[k]];
                    if (q < 0.0) a = (-q) / v;
                }
            }
            val[k] = a;
        }
        adiag = fabs(aii);
    }
    // max |a_ii|: non-negative doubles order like their bit patterns
    __shared__ double wmax[4];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) adiag = fmax(adiag, __shfl_xor_sync(0xffffffffu, adiag, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = adiag;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, wmax[w]);
        if (mx > 0.0) atomicMax(diag_max, (unsigned long long)__double_as_longlong(mx));
    }
}

}  // namespace

cudaError_t launch_transport_matrix(const ElemData &d, const TransportPattern &p, const double *porosity,
                                    const double *sol, double *val, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(p.diag_max, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
    if (p.n_edges > 0)
        k_edge_outflow<<<(unsigned)((p.n_edges + 255) / 256), 256, 0, s>>>(p.n_edges, p.edge_start, p.edge_sides, sol,
                                                                           p.edge_flow);
    if (p.n_el > 0)
        k_transport_rows<<<(unsigned)((p.n_el + 127) / 128), 128, 0, s>>>(d, p.n_el, p.row_ptr, p.kind, p.slot_a,
                                                                          p.slot_b, p.ngh_side, p.edge_flow, porosity,
                                                                          sol, val, p.diag_max);
    return cudaGetLastError();
}

}  // namespace mh
