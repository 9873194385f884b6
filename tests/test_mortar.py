"""Mortar coupling of non-matching 1D and 2D elements (mh_create_mortar, mortar_method P0 and P1
of the reference): a channel of its own nodes lying in a fracture plane, not along the
triangles' sides.

CPU: the plane intersections (each segment is covered by the pieces inside the triangles, and
every piece's local coordinates map to the same point on the master and on the slave); the
layout gains the couplings; bad input is refused.  GPU: the assembled edge system equals the
oracle's double Schur complement plus the restated mortar blocks (1e-14 entrywise, scaled by
the diagonal), and the solution equals the FP64 direct solve of the full MH system with the
mortar blocks in its edge rows."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import mhdarcy
import mortar as OM
import oracle as O
from helpers import oracle_problem
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc
from mhdarcy.mortar import plane_intersections


def channel_case(n=6, segs=7, y=0.37, seed=3):
    """Kuhn cube with a z = 1/2 fracture and a 1D channel along x at (y, 1/2) with its own
    nodes (none shared with the cube); conductivities like the benchmark cases."""
    cube = mhdarcy.cube_mesh(n, [(2, n // 2)])
    nn = len(cube.nodes)
    xs = np.linspace(0.0, 1.0, segs + 1)
    extra = np.column_stack([xs, np.full(segs + 1, y), np.full(segs + 1, 0.5)])
    nodes = np.vstack([cube.nodes, extra])
    seg = np.full((segs, 4), -1, np.int32)
    seg[:, 0] = nn + np.arange(segs)
    seg[:, 1] = nn + np.arange(1, segs + 1)
    mesh = mhdarcy.Mesh(nodes, np.concatenate([cube.el_dim, np.ones(segs, np.int32)]),
                        np.vstack([cube.el_nodes, seg]))
    rng = np.random.default_rng(seed)
    ne = mesh.n_elements
    dim = mesh.el_dim
    K = 10.0 ** rng.normal(-6.0, 1.0, ne)
    delta = np.ones(ne)
    K[dim == 2], delta[dim == 2] = 1e-3, 1e-3
    K[dim == 1], delta[dim == 1] = 1e-2, 1e-4
    return mesh, dict(conductivity=K, cross_section=delta)


def intersections(mesh):
    return plane_intersections(mesh)


def test_plane_intersections_cover_the_channel():
    mesh, _ = channel_case()
    m, s, t, xy = intersections(mesh)
    assert len(m) > 0 and np.all(mesh.el_dim[m] == 1) and np.all(mesh.el_dim[s] == 2)
    for ln in np.unique(m):
        sel = m == ln
        assert abs(np.sum(t[sel, 1] - t[sel, 0]) - 1.0) < 1e-12
    X = mesh.nodes
    for k in range(len(m)):
        P0, P1 = X[mesh.el_nodes[m[k], 0]], X[mesh.el_nodes[m[k], 1]]
        A, B, C = (X[mesh.el_nodes[s[k], j]] for j in range(3))
        for q in range(2):
            pm = P0 + t[k, q] * (P1 - P0)
            ps = A + xy[k, q, 0] * (B - A) + xy[k, q, 1] * (C - A)
            assert np.abs(pm - ps).max() < 1e-12
            assert xy[k, q].min() > -1e-12 and xy[k, q].sum() < 1 + 1e-12


@pytest.mark.parametrize("method", [_lib.MH_MORTAR_P0, _lib.MH_MORTAR_P1])
def test_mortar_layout(method):
    """The edge system's pattern gains the master-slave couplings (host layout, no device
    needed); a pair that is not (1D master, 2D slave) is refused."""
    mesh, _ = channel_case()
    m, s, t, xy = intersections(mesh)
    with mhdarcy.MHSystem(mesh) as a, mhdarcy.MHSystem(mesh, mortar=(method, 1.0, m, s, t, xy)) as b:
        assert b.sizes.schur_nnz > a.sizes.schur_nnz
        assert b.n_edges == a.n_edges
    with pytest.raises(mhdarcy.MHError) as ei:
        mhdarcy.MHSystem(mesh, mortar=(method, 1.0, s, m, t, xy))  # master and slave swapped
    assert ei.value.status == _lib.MH_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("method", [_lib.MH_MORTAR_P0, _lib.MH_MORTAR_P1])
def test_mortar_system_and_solution(gpu, method):
    import scipy.sparse as sp
    mesh, coeffs = channel_case()
    m, s, t, xy = intersections(mesh)
    sigma = 0.7
    with mhdarcy.MHSystem(mesh, mortar=(method, sigma, m, s, t, xy)) as g:
        topo = g.topology()
        bc, _ = dirichlet_x_bc(topo, mesh)
        g.set_coeffs(**coeffs)
        g.set_bc(bc["bc_type"], bc["pressure"])
        g.assemble()
        P = oracle_problem(mesh, topo, g.n_edges, coeffs, bc)
        S, r = O.schur2(P)
        Mo = OM.edge_system_block(mesh, topo, g.n_edges, method, sigma, m, s, t, xy)
        assert abs(Mo).max() > 0
        St = (S + Mo).tocsr()
        rp, col, val, rhs = g.schur_system()
        G = sp.csr_matrix((val, col, rp), shape=St.shape)
        d = np.sqrt(np.abs(St.diagonal()))
        D = sp.diags(1.0 / d)
        assert abs(D @ (G - St) @ D).max() <= 1e-14
        assert np.abs((rhs - r) / d).max() <= 1e-14 * np.abs(r / d).max()
        st = g.solve(method=_lib.MH_SOLVER_PCG64, r_tol=1e-13)
        assert st["status"] in (0, _lib.MH_NOT_CONVERGED) and st["rel_residual"] <= 1e-12, st
        sol = g.solution()
        # the FP64 direct solve of the full MH system with the mortar blocks in its edge rows
        A, b = O.assemble_mh(P)
        off = P.n_sides + P.n_el
        Mmh = OM.mh_matrix_block(mesh, topo, g.n_edges, method, sigma, m, s, t, xy)
        A = A.tolil()
        A[off:, off:] = A[off:, off:] + Mmh
        ref = spla.spsolve(A.tocsc(), b)
        ns, ne = g.n_sides, g.n_elements
        for part in (slice(0, ns), slice(ns, ns + ne), slice(ns + ne, len(ref))):
            assert np.abs(sol[part] - ref[part]).max() <= 1e-8 * np.abs(ref[part]).max()
        # the channel carries flow: the mortar coupling is active
        ch = np.nonzero(mesh.el_dim == 1)[0]
        assert np.abs(sol[ns + ch]).max() > 0


@pytest.mark.parametrize("method", [_lib.MH_MORTAR_P0, _lib.MH_MORTAR_P1])
def test_oracle_mortar_sign_through_both_eliminations(method):
    """The oracle's two views of the mortar terms agree: added to the MH matrix's edge rows
    (the reference's schur0) and solved directly, or added with the opposite sign to the double
    Schur complement (after its scale(-1)) and back-substituted."""
    import scipy.sparse as sp
    mesh, coeffs = channel_case()
    m, s, t, xy = intersections(mesh)
    with mhdarcy.MHSystem(mesh) as g:
        topo, n_edges = g.topology(), g.n_edges
    bc, _ = dirichlet_x_bc(topo, mesh)
    P = oracle_problem(mesh, topo, n_edges, coeffs, bc)
    S, r = O.schur2(P)
    lam = spla.spsolve((S + OM.edge_system_block(mesh, topo, n_edges, method, 0.7, m, s, t, xy)).tocsc(), r)
    sol = O.resolve(P, lam)
    A, b = O.assemble_mh(P)
    off = P.n_sides + P.n_el
    A = A.tolil()
    A[off:, off:] = A[off:, off:] + OM.mh_matrix_block(mesh, topo, n_edges, method, 0.7, m, s, t, xy)
    ref = spla.spsolve(A.tocsc(), b)
    assert np.abs(sol - ref).max() <= 1e-9 * np.abs(ref).max()
