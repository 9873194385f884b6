// The object behind the C ABI's mh_mesh handle: the flat arrays of a mesh and, for a mesh
// read from a gmsh file, the file's node and element ids, element regions and the region
// table (RegionDB, src/mesh/region.cc:107-175).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "topology.hpp"

struct mh_mesh {
    mh::MeshData m;
    bool from_file = false;
    std::vector<int64_t> node_id;          // [n_nodes]
    std::vector<int64_t> el_id;            // [n_el]
    std::vector<int32_t> el_region;        // [n_el] physical id (first tag)
    std::vector<int32_t> el_partition;     // [n_el] third tag, 0 if absent
    std::vector<int64_t> bc_id;            // [n_bc]
    std::vector<int32_t> bc_region;        // [n_bc]
    std::vector<int32_t> region_id;        // region table in order of creation
    std::vector<int32_t> region_dim;
    std::vector<int32_t> region_boundary;
    std::vector<std::string> region_name;
    std::vector<const char *> region_name_ptr;
};
