"""TEST INFRASTRUCTURE ONLY: pure-Python restatement of Flow123d's mesh topology rules, used to
pin the C++ topology builder of the product on small meshes.

Follows Mesh::make_neighbours_and_edges (src/mesh/mesh.cc:343-500), the node-element lists
and set intersections it uses (mesh.cc:265-303), find_lower_dim_element (mesh.cc:306-324),
same_sides (mesh.cc:326-331), element_to_neigh_vb (mesh.cc:660-685) and the side numbering of
RefElement (src/mesh/ref_element.cc:51-76).  Pure Python loops: small meshes only.
"""
import numpy as np

SIDE_NODES = {1: [[0], [1]], 2: [[0, 1], [1, 2], [0, 2]], 3: [[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]]}


def build(mesh):
    dim = [int(d) for d in mesh.el_dim]
    nodes = [[int(v) for v in row[:d + 1]] for row, d in zip(mesh.el_nodes, dim)]
    n_el = len(dim)
    side_start = [0]
    for d in dim:
        side_start.append(side_start[-1] + d + 1)
    node_elements = {}
    for e in range(n_el):
        for v in nodes[e]:
            node_elements.setdefault(v, []).append(e)

    def intersect(ns):
        s = set(node_elements.get(ns[0], []))
        for v in ns[1:]:
            s &= set(node_elements.get(v, []))
        return sorted(s)

    def side_nodes(e, s):
        return sorted(nodes[e][k] for k in SIDE_NODES[dim[e]][s])

    side_edge = [-1] * side_start[-1]
    side_bdr = [-1] * side_start[-1]
    edges = []                 # list of side lists
    bdr_bc, bdr_edge = [], []
    ngh_el, ngh_edge, ngh_side = [], [], []

    bc_dim = [int(d) for d in mesh.bc_dim]
    bc_nodes = [[int(v) for v in row[:d + 1]] for row, d in zip(mesh.bc_nodes, bc_dim)]
    for b, bn in enumerate(bc_nodes):
        lst = [e for e in intersect(bn) if dim[e] == bc_dim[b] + 1]
        if any(dim[e] == bc_dim[b] for e in intersect(bn)):
            raise ValueError("boundary element matches a bulk element of its dimension")
        if not lst:
            continue
        ed = len(edges)
        edges.append([])
        bdr_bc.append(b)
        bdr_edge.append(ed)
        for e in lst:
            for s in range(dim[e] + 1):
                if side_nodes(e, s) == sorted(bn):
                    g = side_start[e] + s
                    edges[ed].append(g)
                    side_edge[g] = ed
                    side_bdr[g] = len(bdr_edge) - 1
                    break

    for e in range(n_el):
        for s in range(dim[e] + 1):
            g = side_start[e] + s
            if side_edge[g] >= 0:
                continue
            sn = side_nodes(e, s)
            cand = intersect(sn)
            same = [o for o in cand if dim[o] == dim[e]]
            lower = [o for o in cand if dim[o] == dim[e] - 1]
            if len(lower) > 1:
                raise ValueError("two lower-dimensional elements match one side")
            is_ngh = len(lower) == 1
            if not is_ngh:
                ed = len(edges)
                edges.append([])
                if len(same) == 1:
                    edges[ed].append(g)
                    side_edge[g] = ed
                    bdr_bc.append(-1)
                    bdr_edge.append(ed)
                    side_bdr[g] = len(bdr_edge) - 1
                    continue
            for o in same:
                for os_ in range(dim[o] + 1):
                    og = side_start[o] + os_
                    if side_edge[og] >= 0 or side_nodes(o, os_) != sn:
                        continue
                    if is_ngh:
                        ne_ = len(edges)
                        edges.append([og])
                        side_edge[og] = ne_
                        ngh_el.append(lower[0])
                        ngh_edge.append(ne_)
                        ngh_side.append(og)
                    else:
                        edges[ed].append(og)
                        side_edge[og] = ed
                    break
    return {
        "el_side_start": np.array(side_start, np.int32),
        "side_edge": np.array(side_edge, np.int32),
        "side_bdr": np.array(side_bdr, np.int32),
        "bdr_bc_element": np.array(bdr_bc, np.int32),
        "bdr_edge": np.array(bdr_edge, np.int32),
        "ngh_element": np.array(ngh_el, np.int32),
        "ngh_edge": np.array(ngh_edge, np.int32),
        "ngh_side": np.array(ngh_side, np.int32),
        "n_edges": len(edges),
        "edge_sides": edges,
    }
