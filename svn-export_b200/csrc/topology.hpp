// Host-side mesh topology of a mixed 1D/2D/3D simplicial mesh, built with the rules of
// Flow123d's Mesh::make_neighbours_and_edges (src/mesh/mesh.cc:343-500) and
// Mesh::element_to_neigh_vb (mesh.cc:660-685).  Everything here is int bookkeeping that
// runs once per mesh; the flat arrays it produces are what the device kernels read.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mh {

// Local node indices of side s of an element of dimension d (src/mesh/ref_element.cc:51-76).
// Tetrahedron side i is the face opposite node i; triangle sides are {0,1},{1,2},{0,2};
// a segment's sides are its end points.
int side_node(int dim, int side, int k);

struct MeshData {
    int64_t n_nodes = 0;
    std::vector<double> xyz;          // [n_nodes*3]
    int64_t n_el = 0;
    std::vector<int32_t> dim;         // [n_el]
    std::vector<int32_t> nodes;       // [n_el*4], -1 padded
    int64_t n_bc = 0;
    std::vector<int32_t> bc_dim;      // [n_bc]
    std::vector<int32_t> bc_nodes;    // [n_bc*4]
};

struct Topology {
    std::vector<int32_t> el_side_start;   // [n_el+1]
    std::vector<int32_t> side_edge;       // [n_sides]
    std::vector<int32_t> side_bdr;        // [n_sides], -1 if not on a boundary object
    std::vector<int32_t> edge_side_start; // [n_edges+1]
    std::vector<int32_t> edge_sides;      // [n_sides] sides of each edge, creation order
    std::vector<int32_t> bdr_bc_el;       // [n_bdr] explicit bc element or -1 (implicit)
    std::vector<int32_t> bdr_edge;        // [n_bdr]
    std::vector<int32_t> ngh_el;          // [n_ngh] lower-dimensional element
    std::vector<int32_t> ngh_edge;        // [n_ngh] edge of the higher-dimensional side
    std::vector<int32_t> ngh_side;        // [n_ngh] that side
    std::vector<int32_t> el_ngh_start;    // [n_el+1] VB neighbours of each (lower) element
    std::vector<int32_t> el_ngh;          // [n_ngh] neighbour indices, creation order
    int64_t n_sides() const { return (int64_t)side_edge.size(); }
    int64_t n_edges() const { return (int64_t)edge_side_start.size() - 1; }
    int64_t n_bdr() const { return (int64_t)bdr_edge.size(); }
    int64_t n_ngh() const { return (int64_t)ngh_el.size(); }
};

// Returns 0 on success; on failure a negative MH_ERR_* code and a message in *err.
int build_topology(const MeshData &m, Topology &t, std::string *err);

// Kuhn (6 tetrahedra per cube) mesh of the unit cube with optional fracture planes and
// 1D channels; see mh_cube_mesh_create in mh_darcy.h for the element order.
int build_cube_mesh(int n, const std::vector<int> &plane_axis, const std::vector<int> &plane_index,
                    const std::vector<int> &line_axis, const std::vector<int> &line_a,
                    const std::vector<int> &line_b, MeshData &m, std::string *err);

}  // namespace mh
