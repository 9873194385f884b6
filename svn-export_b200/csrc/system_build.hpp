// Host construction of the edge-system layout: local edge lists, the symmetric Schur
// pattern, the SELL-C-sigma slot layout, and the element-block -> slot contribution maps.
// Pure integer bookkeeping, done once per mesh.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "mh_darcy.h"
#include "topology.hpp"

namespace mh {

struct HostSystem {
    // instances: element ranges [inst_el[i], inst_el[i+1])
    std::vector<int64_t> inst_el;
    std::vector<int64_t> inst_edge;      // [n_inst+1] edge ranges
    std::vector<int64_t> inst_row;       // [n_inst+1] padded solver-row ranges
    int32_t rows_per_thread = 1;
    int64_t tile_rows = 0;
    int64_t n_rows = 0, n_slices = 0, n_tiles = 0, n_slots = 0, nnz = 0;
    std::vector<int32_t> el_m;           // local block size per element
    std::vector<int64_t> blk_off, rhs_off;
    int64_t n_blk = 0, n_rhs_loc = 0;
    std::vector<int32_t> edge_row, row_edge;
    std::vector<int64_t> row_ptr;        // sorted pattern per solver row (solver-row columns)
    std::vector<int32_t> row_col;
    std::vector<int64_t> slice_off;
    std::vector<int32_t> sell_col;
    std::vector<int32_t> diag_slot;
    std::vector<int32_t> tile_inst;
    // launch plans ([0] FP64 kernels, [1] FP32 kernels): block b works on the tiles
    // [blk_tile_begin[b], blk_tile_end[b]) of instance blk_inst[b]; instance i owns the blocks
    // [inst_blk[i], inst_blk[i+1])
    struct Plan {
        std::vector<int32_t> blk_inst, blk_tile_begin, blk_tile_end, inst_blk;
    } plan[2];
    std::vector<int32_t> slot_cstart, slot_cidx;
    std::vector<int32_t> row_cstart, row_cidx;
    std::vector<int32_t> dim_list[4];
    std::vector<int32_t> csr_slot;       // general systems: SELL slot of every CSR entry
    // constant additions to the edge system (mortar coupling): slots and summed values
    std::vector<int32_t> add_slot;
    std::vector<double> add_val;
};

// Constant couplings added to the edge system besides the element blocks (the mortar terms of
// non-matching lower-dimensional elements): each group is a set of edges that are coupled
// pairwise, with the dense |group| x |group| block of values (row-major) to add.
struct ExtraBlocks {
    std::vector<std::vector<int32_t>> edges;
    std::vector<std::vector<double>> vals;
};

// Local edge list of element e: own side edges then VB-neighbour edges.
int local_edges(const MeshData &m, const Topology &t, int64_t e, int32_t *out);

int build_host_system(const MeshData &m, const Topology &t, const std::vector<int64_t> &inst_el,
                      int rows_per_thread, const int target_blocks[2], HostSystem &hs, std::string *err,
                      const ExtraBlocks *extra = nullptr);

// Layout of a general sparse system given by its CSR pattern (n rows, columns sorted and
// unique in every row, each row holding its diagonal): one instance, rows = unknowns, padded
// to kPadRows, SELL-C-sigma as for the edge system, and csr_slot mapping the CSR entries to
// slots.  No element contributions.
int build_host_system_csr(int64_t n, const int32_t *row_ptr, const int32_t *col, int rows_per_thread,
                          const int target_blocks[2], HostSystem &hs, std::string *err);

// The mortar blocks of mh_create_mortar's intersections (mortar.cpp).
int mortar_blocks(const MeshData &m, const Topology &t, const mh_mortar_desc &d, ExtraBlocks &out, std::string *err);

// Splits every instance's tiles into contiguous runs, one run per block, with about
// target_blocks blocks in total (at least one per instance) in proportion to instance size.
void build_block_plan(HostSystem &hs, int target_blocks, HostSystem::Plan &plan);

// Sets rows per thread (tile = 256 R rows) and rebuilds the tile map and both block plans;
// the matrix layout does not change (instances are padded to kPadRows rows).
void set_launch_shape(HostSystem &hs, int rows_per_thread, const int target_blocks[2]);

}  // namespace mh
