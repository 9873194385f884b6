"""TEST INFRASTRUCTURE ONLY: restatement of the reference's mortar coupling of non-matching 1D
(master) and 2D (slave) elements, the checker of mh_create_mortar.  Never imported by the
product.

Follows, loop for loop:
  * coupling_P0_mortar_assembly     src/flow/darcy_flow_mh.cc:698-799 (mortar_method P0)
  * mh_abstract_assembly_intersection  darcy_flow_mh.cc:815-937 (mortar_method P1)
  * Intersection::intersection_true_size, map_to_master, map_to_slave
                                    src/mesh/intersection.cc
  * Mesh::make_intersec_elements (the master lists)  src/mesh/mesh.cc:758-775
The reference adds its blocks to the MH matrix's edge rows (schur0->mat_set_values); the
returned matrix is what they contribute to the edge system after the final scale(-1), i.e.
their negative.  mh_matrix_block() gives them with the MH matrix's sign.
"""
import numpy as np
import scipy.sparse as sp


def _measure(mesh, e):
    a, b = mesh.el_nodes[e, 0], mesh.el_nodes[e, 1]
    return float(np.linalg.norm(mesh.nodes[b] - mesh.nodes[a]))


def _true_size(mesh, master, master_t):
    # master->measure() * det(master_map) / factorial[1]; master_map = t_Y - t_X (1 x 1)
    return _measure(mesh, master) * (master_t[1] - master_t[0]) / 1.0


def mh_matrix_block(mesh, topo, n_edges, method, sigma, master, slave, master_t, slave_xy):
    """The mortar terms as the reference adds them to the MH matrix (edge rows and columns only),
    as a CSR matrix over the edges."""
    ss, se = topo["el_side_start"], topo["side_edge"]
    edge = lambda e, s: int(se[ss[e] + s])
    I, J, V = [], [], []

    def add(rows, cols, block):
        for a, ra in enumerate(rows):
            for b, cb in enumerate(cols):
                I.append(ra)
                J.append(cb)
                V.append(block[a][b])

    master = np.asarray(master)
    if method == 1:  # P0
        lists = [[] for _ in range(len(mesh.el_dim))]
        for k, m in enumerate(master):
            lists[int(m)].append(k)
        master_map = np.full((1, 2), 0.5)
        slave_map = np.full((1, 3), -1.0 / 3.0)
        for lst in lists:
            if not lst:
                continue
            mi = int(master[lst[0]])
            delta_0 = _measure(mesh, mi)
            for i in range(len(lst) + 1):
                if i == len(lst):
                    delta_i, left_map = delta_0, master_map.T
                    left_idx = [edge(mi, 0), edge(mi, 1)]
                else:
                    k = lst[i]
                    delta_i, left_map = _true_size(mesh, mi, master_t[k]), slave_map.T
                    left_idx = [edge(int(slave[k]), s) for s in range(3)]
                for j in range(len(lst) + 1):
                    if j == len(lst):
                        delta_j, right_map = delta_0, master_map
                        right_idx = [edge(mi, 0), edge(mi, 1)]
                    else:
                        k = lst[j]
                        delta_j, right_map = _true_size(mesh, mi, master_t[k]), slave_map
                        right_idx = [edge(int(slave[k]), s) for s in range(3)]
                    product = -sigma * left_map * delta_i * delta_j @ right_map / delta_0
                    add(left_idx, right_idx, product)
    elif method == 2:  # P1
        base_2D = np.array([[1.0, 0.0, -2.0], [-1.0, 2.0, 2.0], [1.0, -2.0, 0.0]])
        base_1D = np.array([[1.0, -1.0], [0.0, 1.0]])
        for k in range(len(master)):
            mi, si = int(master[k]), int(slave[k])
            # map_to_slave / map_to_master of Y = 1 and X = 0: the points' local coordinates with a
            # leading 1
            p2Y = np.array([1.0, slave_xy[k][1][0], slave_xy[k][1][1]])
            p2X = np.array([1.0, slave_xy[k][0][0], slave_xy[k][0][1]])
            p1Y = np.array([1.0, master_t[k][1]])
            p1X = np.array([1.0, master_t[k][0]])
            dY = np.concatenate([-base_2D @ p2Y, base_1D @ p1Y])
            dX = np.concatenate([-base_2D @ p2X, base_1D @ p1X])
            size = _true_size(mesh, mi, master_t[k])
            A = np.zeros((5, 5))
            for i in range(5):
                for j in range(5):
                    A[i, j] = -sigma * size * (dY[i] * dY[j] + dY[i] * dX[j] / 2 + dX[i] * dY[j] / 2
                                               + dX[i] * dX[j]) * (1.0 / 3.0)
            idx = [edge(si, 0), edge(si, 1), edge(si, 2), edge(mi, 0), edge(mi, 1)]
            add(idx, idx, A)
    M = sp.coo_matrix((V, (I, J)), shape=(n_edges, n_edges)).tocsr()
    M.sum_duplicates()
    return M


def edge_system_block(*args, **kw):
    """The mortar terms' contribution to the edge system (schur2 after scale(-1))."""
    return -mh_matrix_block(*args, **kw)
