// Mesh topology and synthetic Kuhn meshes.  See topology.hpp.
#include "topology.hpp"

#include <algorithm>
#include <cstdio>

#include "mh_darcy.h"

namespace mh {

namespace {
const int kSide1[2][1] = {{0}, {1}};
const int kSide2[3][2] = {{0, 1}, {1, 2}, {0, 2}};
const int kSide3[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};

// Node -> sorted list of bulk elements containing it (Mesh::create_node_element_lists,
// mesh.cc:265-275), stored as CSR.
struct NodeElements {
    std::vector<int64_t> start;
    std::vector<int32_t> el;
};

void build_node_elements(const MeshData &m, NodeElements &ne) {
    ne.start.assign(m.n_nodes + 1, 0);
    for (int64_t e = 0; e < m.n_el; ++e)
        for (int k = 0; k <= m.dim[e]; ++k) ne.start[m.nodes[4 * e + k] + 1]++;
    for (int64_t i = 0; i < m.n_nodes; ++i) ne.start[i + 1] += ne.start[i];
    ne.el.resize(ne.start[m.n_nodes]);
    std::vector<int64_t> fill(ne.start.begin(), ne.start.end() - 1);
    // elements are visited in increasing index, so every list comes out sorted
    for (int64_t e = 0; e < m.n_el; ++e)
        for (int k = 0; k <= m.dim[e]; ++k) ne.el[fill[m.nodes[4 * e + k]]++] = (int32_t)e;
}

// Elements containing every node of `nodes` (Mesh::intersect_element_lists, mesh.cc:278-303).
void intersect(const NodeElements &ne, const int *nodes, int nn, std::vector<int32_t> &out) {
    out.clear();
    if (nn == 0) return;
    out.assign(ne.el.begin() + ne.start[nodes[0]], ne.el.begin() + ne.start[nodes[0] + 1]);
    for (int i = 1; i < nn && !out.empty(); ++i) {
        const int32_t *b = ne.el.data() + ne.start[nodes[i]];
        const int32_t *be = ne.el.data() + ne.start[nodes[i] + 1];
        auto w = std::set_intersection(out.begin(), out.end(), b, be, out.begin());
        out.resize(w - out.begin());
    }
}

// Keep only elements of dimension `dim`; report one of dimension dim-1
// (Mesh::find_lower_dim_element, mesh.cc:306-324).  Returns -2 if two lower-dim match.
int filter_dim(const MeshData &m, std::vector<int32_t> &list, int dim, int32_t *lower) {
    int found = 0;
    size_t w = 0;
    for (size_t i = 0; i < list.size(); ++i) {
        int d = m.dim[list[i]];
        if (d == dim) {
            list[w++] = list[i];
        } else if (d == dim - 1) {
            if (found) return -2;
            found = 1;
            *lower = list[i];
        }
    }
    list.resize(w);
    return found;
}

// Side `s` of element `e` consists of exactly the nodes in `nodes` (Mesh::same_sides,
// mesh.cc:326-331; both lists have dim nodes, so inclusion is equality).
bool same_side(const MeshData &m, int64_t e, int s, const int *nodes, int nn) {
    int d = m.dim[e];
    for (int k = 0; k < d; ++k) {
        int v = m.nodes[4 * e + side_node(d, s, k)];
        bool hit = false;
        for (int j = 0; j < nn; ++j) hit |= (nodes[j] == v);
        if (!hit) return false;
    }
    return true;
}
}  // namespace

int side_node(int dim, int side, int k) {
    switch (dim) {
        case 1: return kSide1[side][k];
        case 2: return kSide2[side][k];
        default: return kSide3[side][k];
    }
}

int build_topology(const MeshData &m, Topology &t, std::string *err) {
    char msg[256];
    t = Topology();
    t.el_side_start.assign(m.n_el + 1, 0);
    for (int64_t e = 0; e < m.n_el; ++e) {
        int d = m.dim[e];
        if (d < 1 || d > 3) {
            snprintf(msg, sizeof msg, "element %lld has unsupported dimension %d", (long long)e, d);
            if (err) *err = msg;
            return MH_ERR_INVALID;
        }
        for (int k = 0; k <= d; ++k) {
            int v = m.nodes[4 * e + k];
            if (v < 0 || v >= m.n_nodes) {
                snprintf(msg, sizeof msg, "element %lld references node %d", (long long)e, v);
                if (err) *err = msg;
                return MH_ERR_INVALID;
            }
        }
        t.el_side_start[e + 1] = t.el_side_start[e] + d + 1;
    }
    const int64_t n_sides = t.el_side_start[m.n_el];
    if (n_sides > INT32_MAX - 1) {
        if (err) *err = "mesh too large for 32-bit side indices";
        return MH_ERR_INVALID;
    }
    t.side_edge.assign(n_sides, -1);
    t.side_bdr.assign(n_sides, -1);
    t.edge_side_start.clear();
    t.edge_side_start.push_back(0);
    t.edge_sides.reserve(n_sides);

    NodeElements ne;
    build_node_elements(m, ne);
    std::vector<int32_t> list;
    list.reserve(64);

    auto new_edge = [&]() {
        t.edge_side_start.push_back(t.edge_side_start.back());
        return (int32_t)(t.edge_side_start.size() - 2);
    };
    auto add_side = [&](int32_t side) {
        t.edge_sides.push_back(side);
        t.edge_side_start.back()++;
    };

    // 1. explicit boundary elements (mesh.cc:358-410)
    for (int64_t b = 0; b < m.n_bc; ++b) {
        int bd = m.bc_dim[b];
        int nn = bd + 1;
        int bn[4];
        for (int k = 0; k < nn; ++k) {
            bn[k] = m.bc_nodes[4 * b + k];
            if (bn[k] < 0 || bn[k] >= m.n_nodes) {
                if (err) *err = "boundary element references an invalid node";
                return MH_ERR_INVALID;
            }
        }
        intersect(ne, bn, nn, list);
        int32_t lower = -1;
        int f = filter_dim(m, list, bd + 1, &lower);
        if (f != 0) {
            snprintf(msg, sizeof msg,
                     "boundary element %lld matches a bulk element of its own dimension",
                     (long long)b);
            if (err) *err = msg;
            return MH_ERR_TOPOLOGY;
        }
        if (list.empty()) continue;  // lonely boundary element: skipped, as in mesh.cc:371-375
        int32_t edge = new_edge();
        int32_t bdr = (int32_t)t.bdr_edge.size();
        t.bdr_edge.push_back(edge);
        t.bdr_bc_el.push_back((int32_t)b);
        for (int32_t e : list) {
            for (int s = 0; s <= m.dim[e]; ++s) {
                if (same_side(m, e, s, bn, nn)) {
                    int32_t side = t.el_side_start[e] + s;
                    add_side(side);
                    t.side_edge[side] = edge;
                    t.side_bdr[side] = bdr;
                    break;
                }
            }
        }
    }

    // 2. sides of bulk elements (mesh.cc:412-497)
    for (int64_t e = 0; e < m.n_el; ++e) {
        int d = m.dim[e];
        for (int s = 0; s <= d; ++s) {
            int32_t side = t.el_side_start[e] + s;
            if (t.side_edge[side] >= 0) continue;
            int sn[3];
            for (int k = 0; k < d; ++k) sn[k] = m.nodes[4 * e + side_node(d, s, k)];
            intersect(ne, sn, d, list);
            int32_t lower = -1;
            int f = filter_dim(m, list, d, &lower);
            if (f < 0) {
                snprintf(msg, sizeof msg,
                         "two lower-dimensional elements match side %d of element %lld", s,
                         (long long)e);
                if (err) *err = msg;
                return MH_ERR_TOPOLOGY;
            }
            bool is_ngh = (f == 1);
            int32_t edge = -1;
            if (!is_ngh) {
                edge = new_edge();
                if (list.size() == 1) {  // outer side: implicit boundary object
                    add_side(side);
                    t.side_edge[side] = edge;
                    int32_t bdr = (int32_t)t.bdr_edge.size();
                    t.bdr_edge.push_back(edge);
                    t.bdr_bc_el.push_back(-1);
                    t.side_bdr[side] = bdr;
                    continue;
                }
            }
            for (int32_t o : list) {
                for (int os = 0; os <= m.dim[o]; ++os) {
                    int32_t oside = t.el_side_start[o] + os;
                    if (t.side_edge[oside] >= 0) continue;
                    if (!same_side(m, o, os, sn, d)) continue;
                    if (is_ngh) {
                        int32_t ne_ = new_edge();
                        add_side(oside);
                        t.side_edge[oside] = ne_;
                        t.ngh_el.push_back(lower);
                        t.ngh_edge.push_back(ne_);
                        t.ngh_side.push_back(oside);
                    } else {
                        add_side(oside);
                        t.side_edge[oside] = edge;
                    }
                    break;
                }
            }
            if (!is_ngh &&
                (size_t)(t.edge_side_start[edge + 1] - t.edge_side_start[edge]) != list.size()) {
                if (err) *err = "some connected sides were not found";
                return MH_ERR_TOPOLOGY;
            }
        }
    }

    // 3. element -> VB neighbours (mesh.cc:660-685)
    const int64_t n_ngh = (int64_t)t.ngh_el.size();
    t.el_ngh_start.assign(m.n_el + 1, 0);
    for (int64_t i = 0; i < n_ngh; ++i) t.el_ngh_start[t.ngh_el[i] + 1]++;
    for (int64_t e = 0; e < m.n_el; ++e) t.el_ngh_start[e + 1] += t.el_ngh_start[e];
    t.el_ngh.resize(n_ngh);
    std::vector<int32_t> fill(t.el_ngh_start.begin(), t.el_ngh_start.end() - 1);
    for (int64_t i = 0; i < n_ngh; ++i) t.el_ngh[fill[t.ngh_el[i]]++] = (int32_t)i;

    for (int64_t s = 0; s < n_sides; ++s) {
        if (t.side_edge[s] < 0) {
            if (err) *err = "a side was left without an edge";
            return MH_ERR_TOPOLOGY;
        }
    }
    return MH_OK;
}

int build_cube_mesh(int n, const std::vector<int> &plane_axis, const std::vector<int> &plane_index,
                    const std::vector<int> &line_axis, const std::vector<int> &line_a,
                    const std::vector<int> &line_b, MeshData &m, std::string *err) {
    if (n < 1 || n > 1024) {
        if (err) *err = "cube resolution out of range";
        return MH_ERR_INVALID;
    }
    const int64_t n1 = n + 1;
    m = MeshData();
    m.n_nodes = n1 * n1 * n1;
    m.xyz.resize(m.n_nodes * 3);
    auto node = [&](int64_t i, int64_t j, int64_t k) { return (int32_t)(i + n1 * (j + n1 * k)); };
    for (int64_t k = 0; k < n1; ++k)
        for (int64_t j = 0; j < n1; ++j)
            for (int64_t i = 0; i < n1; ++i) {
                int64_t v = node(i, j, k);
                m.xyz[3 * v + 0] = (double)i / n;
                m.xyz[3 * v + 1] = (double)j / n;
                m.xyz[3 * v + 2] = (double)k / n;
            }
    for (size_t p = 0; p < plane_axis.size(); ++p)
        if (plane_axis[p] < 0 || plane_axis[p] > 2 || plane_index[p] < 0 || plane_index[p] > n) {
            if (err) *err = "fracture plane out of range";
            return MH_ERR_INVALID;
        }
    for (size_t l = 0; l < line_axis.size(); ++l)
        if (line_axis[l] < 0 || line_axis[l] > 2 || line_a[l] < 0 || line_a[l] > n ||
            line_b[l] < 0 || line_b[l] > n) {
            if (err) *err = "channel out of range";
            return MH_ERR_INVALID;
        }
    const int64_t n_tet = 6 * (int64_t)n * n * n;
    const int64_t n_tri = 2 * (int64_t)n * n * (int64_t)plane_axis.size();
    const int64_t n_seg = (int64_t)n * (int64_t)line_axis.size();
    m.n_el = n_tet + n_tri + n_seg;
    m.dim.resize(m.n_el);
    m.nodes.assign(m.n_el * 4, -1);
    // Kuhn subdivision: one tetrahedron per axis permutation (a,b,c): 000 -> +e_a -> +e_b -> 111.
    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    int64_t e = 0;
    for (int64_t k = 0; k < n; ++k)
        for (int64_t j = 0; j < n; ++j)
            for (int64_t i = 0; i < n; ++i)
                for (int t = 0; t < 6; ++t) {
                    int64_t c[3] = {i, j, k};
                    m.dim[e] = 3;
                    m.nodes[4 * e + 0] = node(c[0], c[1], c[2]);
                    for (int s = 0; s < 2; ++s) {
                        c[perm[t][s]]++;
                        m.nodes[4 * e + 1 + s] = node(c[0], c[1], c[2]);
                    }
                    m.nodes[4 * e + 3] = node(i + 1, j + 1, k + 1);
                    ++e;
                }
    // Fracture triangles: the two Kuhn face triangles of each grid square of the plane;
    // the face diagonal joins the low corner to the high corner.
    for (size_t p = 0; p < plane_axis.size(); ++p) {
        int ax = plane_axis[p];
        int u = (ax + 1) % 3, w = (ax + 2) % 3;
        if (u > w) std::swap(u, w);
        for (int64_t b = 0; b < n; ++b)
            for (int64_t a = 0; a < n; ++a) {
                int64_t c00[3], c10[3], c11[3], c01[3];
                for (int q = 0; q < 3; ++q) c00[q] = c10[q] = c11[q] = c01[q] = 0;
                c00[ax] = c10[ax] = c11[ax] = c01[ax] = plane_index[p];
                c00[u] = a;     c00[w] = b;
                c10[u] = a + 1; c10[w] = b;
                c11[u] = a + 1; c11[w] = b + 1;
                c01[u] = a;     c01[w] = b + 1;
                m.dim[e] = 2;
                m.nodes[4 * e + 0] = node(c00[0], c00[1], c00[2]);
                m.nodes[4 * e + 1] = node(c10[0], c10[1], c10[2]);
                m.nodes[4 * e + 2] = node(c11[0], c11[1], c11[2]);
                ++e;
                m.dim[e] = 2;
                m.nodes[4 * e + 0] = node(c00[0], c00[1], c00[2]);
                m.nodes[4 * e + 1] = node(c01[0], c01[1], c01[2]);
                m.nodes[4 * e + 2] = node(c11[0], c11[1], c11[2]);
                ++e;
            }
    }
    for (size_t l = 0; l < line_axis.size(); ++l) {
        int ax = line_axis[l];
        int u = (ax + 1) % 3, w = (ax + 2) % 3;
        if (u > w) std::swap(u, w);
        for (int64_t a = 0; a < n; ++a) {
            int64_t c0[3], c1[3];
            c0[ax] = a; c1[ax] = a + 1;
            c0[u] = c1[u] = line_a[l];
            c0[w] = c1[w] = line_b[l];
            m.dim[e] = 1;
            m.nodes[4 * e + 0] = node(c0[0], c0[1], c0[2]);
            m.nodes[4 * e + 1] = node(c1[0], c1[1], c1[2]);
            ++e;
        }
    }
    return MH_OK;
}

}  // namespace mh
