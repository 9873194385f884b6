// Constants and plain views shared by host C++ and CUDA code (no device code here).
#pragma once
#include <cstdint>

namespace mh {

constexpr int kMaxNgh1 = 6;        // VB neighbours of a segment (triangle sides on it)
constexpr int kMaxNgh2 = 2;        // VB neighbours of a triangle (coinciding tetrahedron faces)
constexpr int kSliceRowsHost = 32; // SELL-C-sigma chunk height C
constexpr int kTileRowsBase = 256; // rows of one 256-thread block per slice-per-warp
constexpr int kPadRows = 1024;     // instances are padded to a multiple of this many rows

// Read-only device views of the mesh, coefficients and boundary data used by the
// element kernels (assembly, time term, back-substitution).
struct ElemData {
    const double *xyz;            // [n_nodes*3]
    const int32_t *el_nodes;      // [n_el*4]
    const int32_t *el_side_start; // [n_el+1]
    const int32_t *side_edge;     // [n_sides]
    const int32_t *side_bdr;      // [n_sides]
    const int32_t *el_ngh_start;  // [n_el+1]
    const int32_t *el_ngh;        // [n_ngh]
    const int32_t *ngh_edge;      // [n_ngh]
    const int32_t *ngh_hi_el;     // [n_ngh] element owning the higher-dimensional side
    const double *ngh_side_measure;  // [n_ngh]
    // coefficients
    const double *conductivity;   // [n_el]
    const double *anisotropy;     // [n_el*9] or nullptr (identity)
    const double *cross_section;  // [n_el]
    const double *sigma;          // [n_el]
    const double *source;         // [n_el]
    const double *storativity;    // [n_el]
    // boundary objects
    const int32_t *bc_type;
    const double *bc_pressure, *bc_flux, *bc_sigma;
    // unsteady time term
    int32_t time_mode;            // 0 steady, 1 MH (element diagonal), 2 LMH (edge diagonal)
    double dt;
    const double *prev_pressure;  // MH: element pressures of the previous step [n_el]
    const double *prev_edge;      // LMH: edge pressures of the previous step  [n_edges]
};

}  // namespace mh
