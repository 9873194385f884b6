// Device-side data structures shared by the host runtime (mh_handle.cpp) and the CUDA
// translation units.  Plain structs of device pointers; no ownership here.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mh_types.hpp"

namespace mh {

constexpr int kSliceRows = 32;       // SELL-C-sigma chunk height C (one warp, one row per lane)
constexpr int kWarpsPerBlock = 8;    // 256-thread blocks
constexpr int kBlockThreads = kSliceRows * kWarpsPerBlock;
// Per-instance results of the FP64 residual kernel: {r^.r^, sum d r^2, sum d b^2, b^.b^,
// active flag, unused...} (r^ = D^-1/2 r is the Jacobi-scaled residual, d = diag S).
constexpr int kSumStride = 8;
constexpr int kSumActive = 4;

// Per-instance Krylov control block.  One per independent system (one for a single
// mesh, one per realisation in a batch).  Written only by the last block of each kernel
// for that instance (ticket pattern), read by all blocks at kernel entry.
struct InstCtl {
    double rho;        // r.r of the current residual (scaled space)
    double alpha, beta;
    double rr0;        // r.r at (re)start
    double tol2;       // stop when r.r <= tol2
    double rr;         // last r.r
    double scale;      // IR: norm of the outer residual the inner solve was started from
    double aux[3];
    int32_t iter;      // iterations of the current Krylov run
    int32_t max_it;
    int32_t done;      // 1 once converged, stopped or broken down
    int32_t status;    // 0 converged, 1 max_it, -8 breakdown, -6 non-finite
    uint32_t ticket;   // blocks of the current launch that have published their partials
    int32_t pad;
};

// Launch plan of the Krylov kernels: block b works on the tiles [tile_begin[b], tile_end[b])
// of instance blk_inst[b]; instance i owns blocks [inst_blk[i], inst_blk[i+1]).  There is one
// plan per precision because the FP64 and FP32 SpMV kernels fit different block counts per SM.
struct DevPlan {
    int32_t n_blocks = 0;
    int32_t *blk_inst = nullptr, *tile_begin = nullptr, *tile_end = nullptr, *inst_blk = nullptr;
};

// SELL-C-sigma matrix view in solver-row space (rows padded per instance to whole tiles).
template <typename T> struct SellView {
    int64_t n_rows;
    const int64_t *slice_off;  // [n_slices+1] first slot of each 32-row slice
    const int32_t *col;        // [slots]
    const T *val;              // [slots]
};

// Handle-owned device buffers of the edge system and the Krylov work vectors.
struct DevSystem {
    int64_t n_rows = 0, n_slices = 0, n_tiles = 0, n_slots = 0;
    int32_t rows_per_thread = 1;     // R: slices per warp per tile
    int32_t n_inst = 0;
    DevPlan plan[2];                 // [0]: FP64 kernels, [1]: FP32 kernels
    int64_t *slice_off = nullptr;
    int32_t *col = nullptr;
    double *val_raw = nullptr;       // S  (reference schur2 after scale(-1))
    double *val64 = nullptr;         // D^-1/2 S D^-1/2
    float *val32 = nullptr;          // same in FP32
    int32_t *diag_slot = nullptr;    // [n_rows]
    int32_t *row_edge = nullptr;     // [n_rows] edge of each solver row or -1 (padding)
    int32_t *edge_row = nullptr;     // [n_edges]
    int32_t *tile_inst = nullptr;    // [n_tiles]
    double *dsq = nullptr;           // sqrt(diag S) per row
    double *b = nullptr;             // rhs (original scaling)
    double *bh = nullptr;            // D^-1/2 b
    // FP64 Krylov vectors (scaled space)
    double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *w = nullptr;
    // FP32 inner vectors
    float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr, *z32 = nullptr;
    double *partial = nullptr;       // [max plan blocks * 4]
    InstCtl *ctl = nullptr;          // [n_inst]
    int32_t *n_done = nullptr;       // instances finished in the current Krylov run
    double *inst_sums = nullptr;     // [n_inst * 4] results of the residual kernel
    uint32_t *sum_ticket = nullptr;  // [n_inst]
};

// Contribution maps from element-local blocks to SELL slots / solver rows.
struct DevAssembly {
    int64_t n_blk = 0, n_rhs_loc = 0;
    int64_t *blk_off = nullptr;      // [n_el]
    int64_t *rhs_off = nullptr;      // [n_el]
    double *blk = nullptr;           // element-local S2 blocks, m x m row-major
    double *rhs_loc = nullptr;       // element-local r2 entries
    int32_t *slot_cstart = nullptr;  // [n_slots+1]
    int32_t *slot_cidx = nullptr;    // [n_blk]
    int32_t *row_cstart = nullptr;   // [n_rows+1]
    int32_t *row_cidx = nullptr;     // [n_rhs_loc]
    int32_t *dim_list[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t dim_count[4] = {0, 0, 0, 0};
    int32_t *status = nullptr;       // bit 0: singular local matrix, bit 1: non-finite value
    int64_t n_add = 0;               // constant additions to the edge system (mortar terms)
    int32_t *add_slot = nullptr;
    double *add_val = nullptr;
};

// ---- launchers (assembly.cu) ----
// K1 with `group` elements per block (one per thread; 64, 128 or 256, else 128).
cudaError_t launch_local_blocks(const ElemData &d, const DevAssembly &a, int mode, int group, cudaStream_t s);
cudaError_t launch_gather(const DevAssembly &a, const DevSystem &sys, int mode, cudaStream_t s);
cudaError_t launch_scale(const DevSystem &sys, int matrix, cudaStream_t s);
cudaError_t launch_backsub(const ElemData &d, const DevAssembly &a, const DevSystem &sys, double *sol,
                           int64_t n_sides, int64_t n_el, int64_t n_edges, cudaStream_t s);
// Darcy flux vector at every element centre from the side fluxes in sol (postprocess.cu):
// out[3 e + k], k = x, y, z.
cudaError_t launch_element_flux(const ElemData &d, const DevAssembly &a, const double *sol, double *out,
                                cudaStream_t s);
// Pressure at every node from the element and side pressures of sol (postprocess.cu): one
// thread per node over its elements, inc_start [n_nodes+1] / inc_el (ascending element ids).
cudaError_t launch_node_pressure(const ElemData &d, const int32_t *inc_start, const int32_t *inc_el, int64_t n_nodes,
                                 const double *sol, int64_t n_sides, int64_t n_el, double *out, cudaStream_t s);
// Convection matrix of the explicit transport (transport.cu).  The pattern is built on the host
// once per mesh: per row, slots sorted by column, each with its kind and the side indices its
// value reads (edge: own side a, other side b; VB: the higher-dimensional side a).
constexpr int kTrDiag = 0, kTrEdge = 1, kTrVbLower = 2, kTrVbHigher = 3;
struct TransportPattern {
    int64_t n_el = 0, n_edges = 0, nnz = 0;
    int32_t *row_ptr = nullptr, *kind = nullptr, *slot_a = nullptr, *slot_b = nullptr;  // device
    int32_t *edge_start = nullptr, *edge_sides = nullptr, *ngh_side = nullptr;          // device
    double *edge_flow = nullptr;                                                         // [n_edges]
    unsigned long long *diag_max = nullptr;                                              // max |a_ii| bits
};
// val [nnz] in the pattern's slot order; porosity [n_el] on the device or null (1).
cudaError_t launch_transport_matrix(const ElemData &d, const TransportPattern &p, const double *porosity,
                                    const double *sol, double *val, cudaStream_t s);

// Water balance per region (postprocess.cu).  Items grouped by region (ascending within a
// region) and cut into chunks: *_chunk_begin [n_chunks+1] into *_items, *_region_chunk
// [n_reg+1] into the chunks.  Device arrays, built on the host for each call.
struct BalanceLists {
    const int32_t *bdr_items = nullptr, *src_items = nullptr;           // side / element ids
    const int64_t *bdr_chunk_begin = nullptr, *src_chunk_begin = nullptr;
    const int64_t *bdr_region_chunk = nullptr, *src_region_chunk = nullptr;
    int64_t n_bdr_chunks = 0, n_src_chunks = 0;
    int32_t n_bdr_reg = 0, n_src_reg = 0;
};
// bdr_out [3 n_bdr_reg] total, outflow, inflow of the boundary side fluxes; src_out
// [n_src_reg] the sources; partial holds 3 n_bdr_chunks + n_src_chunks values.
cudaError_t launch_water_balance(const ElemData &d, const double *sol, const BalanceLists &L, double *partial,
                                 double *bdr_out, double *src_out, cudaStream_t s);
constexpr int64_t kBalanceChunkItems = 8192;

// x = lambda * dsq (initial guess in scaled space; padding rows 0).
cudaError_t launch_scale_in(const DevSystem &sys, const double *lambda, cudaStream_t s);

// ---- launchers (solver.cu) ----
// Krylov kernels on the scaled system; `prec` = 64 or 32.
// FP64 CG start from sys.x: tol2 = max(rtol2 * |bh|^2, atol2); with use_active only the
// instances flagged in inst_sums[4i+3] run.
cudaError_t launch_cg_init(const DevSystem &sys, double rtol2, double atol2, int max_it, int use_active,
                           cudaStream_t s);
cudaError_t launch_cg_iteration(const DevSystem &sys, int prec, cudaStream_t s);
cudaError_t launch_cg_spmv(const DevSystem &sys, int prec, cudaStream_t s);
cudaError_t launch_cg_update(const DevSystem &sys, int prec, cudaStream_t s);
// r = bh - S64 x (FP64) and per-instance sums {sum r^2, sum d r^2, sum d bh^2}.
cudaError_t launch_residual64(const DevSystem &sys, cudaStream_t s);
// IR helpers: start an FP32 inner solve from r; fold its correction back into x.
cudaError_t launch_ir_start(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s);
cudaError_t launch_ir_correct(const DevSystem &sys, cudaStream_t s);
// Reliable update: continue the FP32 recursion from the recomputed FP64 residual, keeping p.
cudaError_t launch_ir_replace(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s);
cudaError_t launch_ir_continue(const DevSystem &sys, double rtol2, int max_it, cudaStream_t s);
cudaError_t launch_reset_ctl(const DevSystem &sys, cudaStream_t s);
// Device-side loop control for a conditional WHILE node: init (before the node) resets the body
// count loop[0]; next (the body's last kernel) counts the body and keeps the loop running while
// an instance is not done and the count is below loop[1].
cudaError_t launch_loop_init(const DevSystem &sys, cudaGraphConditionalHandle hnd, int32_t *loop, cudaStream_t s);
cudaError_t launch_loop_next(const DevSystem &sys, cudaGraphConditionalHandle hnd, int32_t *loop, cudaStream_t s);
// Blocks per Krylov launch for precision 64 or 32: SMs of the current device times the blocks
// of that precision's SpMV kernel that fit on one SM (148 x 4 without a device).
int krylov_target_blocks(int rows_per_thread, int prec);

}  // namespace mh
