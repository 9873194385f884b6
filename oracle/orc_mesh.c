/*
 * orc_mesh.c -- TEST INFRASTRUCTURE ONLY.  Plain-C restatement of Flow123d's mesh topology
 * rules, so that bench.py's CPU arm (and the tests) can build a problem without the GPU
 * library.  It is never linked into or called by the product.
 *
 * Follows, like oracle/topology.py (the pure-Python restatement it is checked against):
 *   Mesh::make_neighbours_and_edges   src/mesh/mesh.cc:343-500
 *     (boundary elements first, :363-399; then every unassigned element side, :401-497)
 *   node-element lists and their intersections   mesh.cc:265-303
 *   find_lower_dim_element                       mesh.cc:306-324
 *   same_sides                                   mesh.cc:326-331
 *   element_to_neigh_vb                          mesh.cc:660-685
 *   side numbering of RefElement                 src/mesh/ref_element.cc:51-76
 *
 * Build: make -C oracle (into libmhoracle.so with mh_oracle.c).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const int TOPO_SIDE_1[2][1] = {{0}, {1}};
static const int TOPO_SIDE_2[3][2] = {{0, 1}, {1, 2}, {0, 2}};
static const int TOPO_SIDE_3[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};

static int topo_side_node(int dim, int s, int k) {
    return dim == 1 ? TOPO_SIDE_1[s][k] : dim == 2 ? TOPO_SIDE_2[s][k] : TOPO_SIDE_3[s][k];
}

static void sort_small(int32_t *a, int n) {
    for (int i = 1; i < n; ++i)
        for (int j = i; j > 0 && a[j - 1] > a[j]; --j) {
            int32_t t = a[j];
            a[j] = a[j - 1];
            a[j - 1] = t;
        }
}

typedef struct {
    int64_t n_el;
    const int32_t *dim, *nodes;
    const int64_t *ne_start;   /* node -> elements (ascending), CSR */
    const int32_t *ne_list;
} topo_ctx;

/* sorted node ids of side s of element e (dim nodes) */
static void side_nodes(const topo_ctx *T, int64_t e, int s, int32_t *out) {
    const int d = T->dim[e];
    for (int k = 0; k < d; ++k) out[k] = T->nodes[4 * e + topo_side_node(d, s, k)];
    sort_small(out, d);
}

/* Elements containing all nodes ns[0..k) in ascending order (the intersection of the
 * node-element lists); returns the count, of which the first cap are stored. */
static int intersect(const topo_ctx *T, const int32_t *ns, int k, int32_t *out, int cap) {
    int best = 0;
    for (int i = 1; i < k; ++i)
        if (T->ne_start[ns[i] + 1] - T->ne_start[ns[i]] < T->ne_start[ns[best] + 1] - T->ne_start[ns[best]]) best = i;
    int cnt = 0;
    for (int64_t p = T->ne_start[ns[best]]; p < T->ne_start[ns[best] + 1]; ++p) {
        const int32_t e = T->ne_list[p];
        int all = 1;
        for (int i = 0; i < k && all; ++i) {
            if (i == best) continue;
            int64_t lo = T->ne_start[ns[i]], hi = T->ne_start[ns[i] + 1];
            while (lo < hi) {
                int64_t mid = (lo + hi) / 2;
                if (T->ne_list[mid] < e) lo = mid + 1; else hi = mid;
            }
            all = lo < T->ne_start[ns[i] + 1] && T->ne_list[lo] == e;
        }
        if (all) {
            if (cnt < cap) out[cnt] = e;
            ++cnt;
        }
    }
    return cnt;
}

/* Topology of a mixed 1D/2D/3D simplicial mesh: element sides, edges (groups of coincident
 * sides), boundary objects and VB neighbours, in the creation order of the reference.
 * Inputs: el_dim [n_el] (1..3), el_nodes [4 n_el]; bc_dim [n_bc] (0..2), bc_nodes [4 n_bc].
 * Outputs (caller-allocated): el_side_start [n_el+1], side_edge and side_bdr [n_sides],
 * bdr_bc_element and bdr_edge [n_sides + n_bc], ngh_element / ngh_edge / ngh_side [n_sides];
 * counts[0..2] = edges, boundary objects, neighbours.  Returns 0, -7 when the mesh breaks a
 * rule of the reference (two lower-dimensional elements on one side, a boundary element
 * matching a bulk element of its own dimension), or -1 when more than 1024 elements share a
 * side's nodes. */
int orc_topology(int64_t n_nodes, int64_t n_el, const int32_t *el_dim, const int32_t *el_nodes, int64_t n_bc,
                 const int32_t *bc_dim, const int32_t *bc_nodes, int32_t *el_side_start, int32_t *side_edge,
                 int32_t *side_bdr, int32_t *bdr_bc_element, int32_t *bdr_edge, int32_t *ngh_element,
                 int32_t *ngh_edge, int32_t *ngh_side, int64_t *counts) {
    int64_t *ne_start = (int64_t *)calloc((size_t)n_nodes + 1, sizeof(int64_t));
    el_side_start[0] = 0;
    for (int64_t e = 0; e < n_el; ++e) {
        el_side_start[e + 1] = el_side_start[e] + el_dim[e] + 1;
        for (int k = 0; k <= el_dim[e]; ++k) ne_start[el_nodes[4 * e + k] + 1]++;
    }
    for (int64_t v = 0; v < n_nodes; ++v) ne_start[v + 1] += ne_start[v];
    int32_t *ne_list = (int32_t *)malloc((size_t)(ne_start[n_nodes] + 1) * sizeof(int32_t));
    int64_t *fill = (int64_t *)malloc((size_t)(n_nodes + 1) * sizeof(int64_t));
    memcpy(fill, ne_start, (size_t)(n_nodes + 1) * sizeof(int64_t));
    for (int64_t e = 0; e < n_el; ++e)
        for (int k = 0; k <= el_dim[e]; ++k) ne_list[fill[el_nodes[4 * e + k]]++] = (int32_t)e;
    free(fill);
    const int64_t n_sides = el_side_start[n_el];
    for (int64_t g = 0; g < n_sides; ++g) side_edge[g] = side_bdr[g] = -1;
    topo_ctx T = {n_el, el_dim, el_nodes, ne_start, ne_list};
    int64_t n_edges = 0, n_bdr = 0, n_ngh = 0;
    int rc = 0;
    enum { CAP = 1024 };
    int32_t cand[CAP];

    /* explicit boundary elements (mesh.cc:363-399) */
    for (int64_t b = 0; b < n_bc && !rc; ++b) {
        const int bd = bc_dim[b];
        int32_t bn[4];
        for (int k = 0; k <= bd; ++k) bn[k] = bc_nodes[4 * b + k];
        sort_small(bn, bd + 1);
        const int nc = intersect(&T, bn, bd + 1, cand, CAP);
        if (nc > CAP) {
            rc = -1;
            break;
        }
        int n_up = 0;
        for (int i = 0; i < nc; ++i) {
            if (el_dim[cand[i]] == bd) rc = -7;
            if (el_dim[cand[i]] == bd + 1) ++n_up;
        }
        if (rc || n_up == 0) continue;
        const int64_t ed = n_edges++;
        bdr_bc_element[n_bdr] = (int32_t)b;
        bdr_edge[n_bdr] = (int32_t)ed;
        ++n_bdr;
        for (int i = 0; i < nc; ++i) {
            const int32_t e = cand[i];
            if (el_dim[e] != bd + 1) continue;
            for (int s = 0; s <= el_dim[e]; ++s) {
                int32_t sn[3];
                side_nodes(&T, e, s, sn);
                if (memcmp(sn, bn, (size_t)(bd + 1) * sizeof(int32_t)) == 0) {
                    const int64_t g = el_side_start[e] + s;
                    side_edge[g] = (int32_t)ed;
                    side_bdr[g] = (int32_t)(n_bdr - 1);
                    break;
                }
            }
        }
    }

    /* element sides in element order (mesh.cc:401-497) */
    for (int64_t e = 0; e < n_el && !rc; ++e) {
        const int d = el_dim[e];
        for (int s = 0; s <= d && !rc; ++s) {
            const int64_t g = el_side_start[e] + s;
            if (side_edge[g] >= 0) continue;
            int32_t sn[3];
            side_nodes(&T, e, s, sn);
            const int nc = intersect(&T, sn, d, cand, CAP);
            if (nc > CAP) {
                rc = -1;
                break;
            }
            int n_same = 0, n_lower = 0;
            int32_t lower = -1;
            for (int i = 0; i < nc; ++i) {
                if (el_dim[cand[i]] == d) ++n_same;
                if (el_dim[cand[i]] == d - 1) {
                    ++n_lower;
                    lower = cand[i];
                }
            }
            if (n_lower > 1) {
                rc = -7;
                break;
            }
            const int is_ngh = n_lower == 1;
            int64_t ed = -1;
            if (!is_ngh) {
                ed = n_edges++;
                if (n_same == 1) {
                    side_edge[g] = (int32_t)ed;
                    bdr_bc_element[n_bdr] = -1;
                    bdr_edge[n_bdr] = (int32_t)ed;
                    side_bdr[g] = (int32_t)n_bdr;
                    ++n_bdr;
                    continue;
                }
            }
            for (int i = 0; i < nc; ++i) {
                const int32_t o = cand[i];
                if (el_dim[o] != d) continue;
                for (int os = 0; os <= d; ++os) {
                    const int64_t og = el_side_start[o] + os;
                    if (side_edge[og] >= 0) continue;
                    int32_t on[3];
                    side_nodes(&T, o, os, on);
                    if (memcmp(on, sn, (size_t)d * sizeof(int32_t)) != 0) continue;
                    if (is_ngh) {
                        const int64_t ne_ = n_edges++;
                        side_edge[og] = (int32_t)ne_;
                        ngh_element[n_ngh] = lower;
                        ngh_edge[n_ngh] = (int32_t)ne_;
                        ngh_side[n_ngh] = (int32_t)og;
                        ++n_ngh;
                    } else {
                        side_edge[og] = (int32_t)ed;
                    }
                    break;
                }
            }
        }
    }
    free(ne_start);
    free(ne_list);
    counts[0] = n_edges;
    counts[1] = n_bdr;
    counts[2] = n_ngh;
    return rc;
}
