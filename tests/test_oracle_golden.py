"""Pins the CPU oracle to the reference's own golden outputs (no GPU).

t01: raw_output.txt of tests/01_steady_flow_123d, printed with %.8g after a PETSc CG solve to
rtol 1e-10, so agreement is expected at the printing precision.  t05/t06/t10: element
pressures of the reference's VTK outputs, solved with the reference's default tolerances
(r_tol 1e-7), so agreement is expected at that level.  t06 also has analytic answers."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
import topology as T
from helpers import fixture_bc, fixture_coeffs, load_fixture, oracle_problem


def problem(name, **kw):
    z, mesh = load_fixture(name)
    topo = T.build(mesh)
    P = oracle_problem(mesh, topo, topo["n_edges"], fixture_coeffs(z), fixture_bc(z, topo), **kw)
    return z, mesh, topo, P


def test_t01_raw_output():
    z, mesh, topo, P = problem("t01")
    sol = O.solve_mh_direct(P)
    ns, ne = P.n_sides, P.n_el
    assert np.array_equal(z["ref_el_id"], z["el_id"])
    p = sol[ns:ns + ne]
    # the reference solved to PETSc rtol 1e-10 and printed %.8g: agreement to ~5e-9 absolute
    tol = lambda ref: 1e-8 + 5e-9 * np.abs(ref)
    assert np.all(np.abs(p - z["ref_pressure"]) <= tol(z["ref_pressure"]))
    ss, se = topo["el_side_start"], topo["side_edge"]
    lam = sol[ns + ne:]
    for e in range(ne):
        n = z["el_dim"][e] + 1
        assert z["ref_n_sides"][e] == n
        sp = lam[se[ss[e]:ss[e] + n]]
        sf = sol[ss[e]:ss[e] + n]
        np.testing.assert_array_less(np.abs(sp - z["ref_side_pressure"][e, :n]), tol(z["ref_side_pressure"][e, :n]))
        np.testing.assert_array_less(np.abs(sf - z["ref_side_flux"][e, :n]), tol(z["ref_side_flux"][e, :n]))


def test_t01_element_flux_vectors():
    """Element-centre flux vectors (the raw_output's three flux columns) of every element of
    t01: lines, triangles and tetrahedra, at the printing precision."""
    z, mesh, topo, P = problem("t01")
    u = O.element_flux(P, O.solve_mh_direct(P))
    ref = z["ref_flux"]
    assert u.shape == ref.shape
    assert set(np.unique(z["el_dim"])) == {1, 2, 3}
    assert np.all(np.abs(u - ref) <= 1e-8 + 5e-9 * np.abs(ref))


def fixture_regions(z, topo):
    """Region indices of a fixture's boundary objects (through their boundary elements, so
    every boundary object must have one) and elements, and the region ids in index order."""
    bids = sorted(set(z["bc_region"].tolist()))
    eids = sorted(set(z["el_region"].tolist()))
    bdr = np.array([bids.index(z["bc_region"][b]) for b in topo["bdr_bc_element"]], np.int32)
    el = np.array([eids.index(r) for r in z["el_region"]], np.int32)
    return bdr, el, bids, eids


def test_t01_node_pressures():
    """Node pressures of the output mesh ($NodeData "pressure_nodes_[L]", printed %g)."""
    z, mesh, topo, P = problem("t01")
    p = O.node_pressure(P, O.solve_mh_direct(P))
    ref = z["ref_node_pressure"]
    assert p.shape == ref.shape
    assert np.all(np.abs(p - ref) <= 5e-6 * np.abs(ref) + 1e-10)


def test_t01_water_balance():
    """The boundary table of water_balance.out (printed %g): per boundary region the total,
    outflow and inflow; the totals are differences of flows of about 1, so they also carry the
    reference solver's own 1e-10 tolerance.  t01 has no sources."""
    z, mesh, topo, P = problem("t01")
    assert np.all(topo["bdr_bc_element"] >= 0)  # every boundary object has its element
    bdr, el, bids, eids = fixture_regions(z, topo)
    ob, osrc = O.water_balance(P, O.solve_mh_direct(P), bdr, el)
    scale = np.abs(z["ref_bdr_balance"][:, 1:]).max()
    for rid, *vals in z["ref_bdr_balance"]:
        got = ob[bids.index(int(rid))]
        assert np.all(np.abs(got - vals) <= 5e-6 * np.abs(vals) + 1e-9 * scale), (rid, got, vals)
    assert np.allclose(ob[:, 0], ob[:, 1] + ob[:, 2], rtol=0, atol=1e-15 * scale)
    for rid, val in z["ref_src_balance"]:
        assert osrc[eids.index(int(rid))] == val == 0.0


def test_t08_sources():
    """tests/08_steady_flow_sources: a source field given by a formula (evaluated at element
    centres), homogeneous Dirichlet on a square.  Element pressures, node pressures and element
    velocities of the VTK output (solver accuracy 1e-7), and the source table of
    water_balance.txt.  Its boundary table (10.5912) is not reproduced: the same file's source
    total is 10.6684, the fluxes that reproduce its VTK velocities to 1e-10 carry exactly that
    total out through the boundary, and the file's name differs from the other tests' balance
    files; the check here is that the boundary outflow equals the sources."""
    z, mesh, topo, P = problem("t08")
    sol = O.solve_mh_direct(P)
    ns, ne = P.n_sides, P.n_el
    assert np.abs(sol[ns:ns + ne] - z["ref_pressure"]).max() < 1e-8
    assert np.abs(O.node_pressure(P, sol) - z["ref_node_pressure"]).max() < 1e-8
    assert np.abs(O.element_flux(P, sol) - z["ref_flux"]).max() < 1e-8
    ob, osrc = O.water_balance(P, sol, np.zeros(len(topo["bdr_bc_element"]), np.int32), np.zeros(ne, np.int32))
    assert abs(osrc[0] - z["ref_src_balance"][0, 1]) <= 5e-6 * abs(osrc[0])
    assert abs(ob[0, 0] - osrc[0]) <= 1e-12 * osrc[0] and ob[0, 2] == 0.0


def test_t03_channel_network():
    """tests/03_transport_small_12d, flow part: 1D channels (conductivity 10) on edges of a 2D
    square (conductivity 1), three channels meeting at one junction edge, channel ends on the
    boundary as point elements, Dirichlet p = x + y everywhere on the boundary.  The VTK output
    has 16 digits; the reference's CG stopped at a preconditioned relative residual of 1e-12,
    which leaves errors of a few 1e-9 in pressures of about 1 and a few 1e-8 in velocities of
    up to 16.  The water balance (printed %g) has regions with both outflow and inflow."""
    z, mesh, topo, P = problem("t03")
    assert set(np.unique(z["el_dim"])) == {1, 2} and set(np.unique(z["bc_dim"])) == {0, 1}
    assert len(topo["ngh_element"]) > 0                         # VB couplings present
    ss, se = topo["el_side_start"], topo["side_edge"]
    assert np.bincount(se[:ss[-1]]).max() >= 3                  # the junction edge
    sol = O.solve_mh_direct(P)
    ns, ne = P.n_sides, P.n_el
    assert np.abs(sol[ns:ns + ne] - z["ref_pressure"]).max() < 1e-8
    assert np.abs(O.node_pressure(P, sol) - z["ref_node_pressure"]).max() < 1e-8
    assert np.abs(O.element_flux(P, sol) - z["ref_flux"]).max() < 1e-7
    assert np.all(topo["bdr_bc_element"] >= 0)
    bdr, el, bids, eids = fixture_regions(z, topo)
    ob, osrc = O.water_balance(P, sol, bdr, el)
    scale = np.abs(z["ref_bdr_balance"][:, 1:]).max()
    mixed = 0
    for rid, *vals in z["ref_bdr_balance"]:
        got = ob[bids.index(int(rid))]
        assert np.all(np.abs(got - vals) <= 5e-6 * np.abs(vals) + 1e-12 * scale), (rid, got, vals)
        mixed += vals[1] > 0 and vals[2] < 0
    assert mixed == 2
    for rid, val in z["ref_src_balance"]:
        assert osrc[eids.index(int(rid))] == val == 0.0


def legacy_problem(name):
    """A fixture whose boundary conditions come from a legacy side-based .fbc file: each
    condition names an element and a local side, whose boundary object gets the condition; the
    other boundary objects have none (no flux)."""
    z, mesh = load_fixture(name)
    topo = T.build(mesh)
    nb = len(topo["bdr_edge"])
    bt, bp = np.zeros(nb, np.int32), np.zeros(nb)
    ss, sb = topo["el_side_start"], topo["side_bdr"]
    for e, s, typ, val in zip(z["lbc_element"], z["lbc_side"], z["lbc_type"], z["lbc_value"]):
        b = sb[ss[e] + s]
        assert b >= 0
        bt[b], bp[b] = typ, val
    P = oracle_problem(mesh, topo, topo["n_edges"], fixture_coeffs(z), {"bc_type": bt, "pressure": bp})
    return z, mesh, topo, P


def test_t02_legacy_network():
    """tests/02_transport_12d, flow part: a 1D network (anisotropy 10) on edges of a 2D domain,
    20 Dirichlet conditions from the legacy .fbc file, solver r_tol 1e-12.  Element and node
    pressures and element velocities of test2.msh are printed with 6 digits; the water balance
    has one region, IMPLICIT BOUNDARY, whose total is the reference solver's residual."""
    z, mesh, topo, P = legacy_problem("t02")
    assert set(np.unique(z["el_dim"])) == {1, 2} and len(topo["ngh_element"]) > 0
    sol = O.solve_mh_direct(P)
    ns, ne = P.n_sides, P.n_el
    printed = lambda got, ref, floor: np.all(np.abs(got - ref) <= 5e-6 * np.abs(ref) + floor * np.abs(ref).max())
    assert printed(sol[ns:ns + ne], z["ref_pressure"], 1e-9)
    assert printed(O.node_pressure(P, sol), z["ref_node_pressure"], 1e-9)
    # the smallest velocities carry the reference solver's error (up to 5.5e-7 on values of 0.006,
    # 4e-8 of the largest velocity) beyond their printing precision
    assert printed(O.element_flux(P, sol), z["ref_flux"], 1e-7)
    ob, osrc = O.water_balance(P, sol, np.zeros(len(topo["bdr_edge"]), np.int32), np.zeros(ne, np.int32))
    (rid, total, out, inflow), = z["ref_bdr_balance"]
    assert rid == -3 and abs(ob[0, 1] - out) <= 5e-6 * out and abs(ob[0, 2] - inflow) <= 5e-6 * out
    assert abs(ob[0, 0]) <= 1e-12 * out and abs(total) < 1e-6 * out
    assert np.all(z["ref_src_balance"][:, 1] == 0.0) and osrc[0] == 0.0


@pytest.mark.parametrize("name", ["t05_dirichlet", "t05_neumann", "t05_robin", "t06_32", "t06_21"])
def test_water_balance_tables(name):
    """The boundary and source tables of water_balance.out of tests 05 (Dirichlet, Neumann,
    Robin) and 06 (3D-2D and 2D-1D coupling with sources): printed %g after solves to the
    reference's r_tol 1e-7, so each entry agrees at its printing plus 2e-6 of the table's
    largest entry (the reference's own spurious flows reach 2.9e-6 on 50)."""
    z, mesh, topo, P = problem(name)
    assert np.all(topo["bdr_bc_element"] >= 0)
    bdr, el, bids, eids = fixture_regions(z, topo)
    ob, osrc = O.water_balance(P, O.solve_mh_direct(P), bdr, el)
    scale = max(np.abs(z["ref_bdr_balance"][:, 1:]).max(), np.abs(z["ref_src_balance"][:, 1]).max())
    close = lambda got, ref: np.all(np.abs(np.asarray(got) - ref) <= 5e-6 * np.abs(ref) + 2e-6 * scale)
    for rid, *vals in z["ref_bdr_balance"]:
        assert close(ob[bids.index(int(rid))], vals), (rid, ob[bids.index(int(rid))], vals)
    for rid, val in z["ref_src_balance"]:
        assert close(osrc[eids.index(int(rid))], val), (rid, osrc[eids.index(int(rid))], val)
    assert abs(ob[:, 0].sum() - osrc.sum()) <= 1e-12 * scale  # what the sources give leaves through the boundary


def test_t01_schur_path_equals_direct():
    z, mesh, topo, P = problem("t01")
    full = O.solve_mh_direct(P)
    via_schur, S, r = O.solve_schur_direct(P)
    assert np.abs(full - via_schur).max() <= 1e-12 * np.abs(full).max()
    # S2 is symmetric positive definite
    assert abs(S - S.T).max() <= 1e-14 * abs(S).max()
    assert np.all(S.diagonal() > 0)


@pytest.mark.parametrize("name", ["t05_dirichlet", "t05_neumann", "t05_robin"])
def test_t05_boundary_conditions(name):
    z, mesh, topo, P = problem(name)
    sol = O.solve_mh_direct(P)
    p = sol[P.n_sides:P.n_sides + P.n_el]
    assert np.abs(p - z["ref_pressure"]).max() < 1e-6
    # the exact solution u = xy is approximated
    c = mesh.centres()
    assert np.abs(p - c[:, 0] * c[:, 1]).max() < 2e-2


def test_t06_coupling_known_answers():
    z, mesh, topo, P = problem("t06_32")
    sol = O.solve_mh_direct(P)
    p = sol[P.n_sides:P.n_sides + P.n_el]
    assert np.abs(p - z["ref_pressure"]).max() < 1e-7
    d2 = mesh.el_dim == 2
    head = p[d2] + mesh.centres()[d2, 2]
    assert np.abs(head + 3.0).max() < 1e-12                        # p2 = -3 (piezometric head)
    z, mesh, topo, P = problem("t06_21")
    sol = O.solve_mh_direct(P)
    p = sol[P.n_sides:P.n_sides + P.n_el]
    assert np.abs(p - z["ref_pressure"]).max() < 1e-6
    assert np.abs(p[mesh.el_dim == 1] + 2.5).max() < 1e-12         # p1 = -2.5


def test_t10_unsteady_mh():
    z, mesh, topo, P = problem("t10_mh", time_mode=1, dt=float(z_dt()))
    prev = np.zeros(P.mh_size)
    prev[P.n_sides:P.n_sides + P.n_el] = z["init_pressure"]
    for step in range(1, 51):
        P.set_prev(prev)
        prev = O.solve_mh_direct(P)
        if step % 10 == 0:
            ref = z["ref_pressure_steps"][step // 10]
            p = prev[P.n_sides:P.n_sides + P.n_el]
            assert np.abs(p - ref).max() < 1e-7 * np.abs(ref).max() * 100


def test_t10_unsteady_lmh():
    """The lumped mixed-hybrid scheme (DarcyFlowLMH_Unsteady, darcy_flow_mh.cc:1695-1827;
    tests/10_unsteady_2d flow_LMH.con): 50 implicit steps from zero, element pressures of the
    VTK output every 10 steps, through the full saddle-point solve and through the double
    Schur complement.  The lumped and consistent schemes differ by up to 1.6% here; the oracle's
    lumped scheme matches the reference's to 1e-9 of the largest pressure."""
    z, mesh, topo, P = problem("t10_lmh", time_mode=2, dt=0.01)
    assert float(z["dt"]) == 0.01  # the fixture's step
    zm, _ = load_fixture("t10_mh")
    import scipy.sparse.linalg as spla
    for via in ("direct", "schur"):
        prev = np.zeros(P.mh_size)
        for step in range(1, 51):
            P.set_prev(prev)
            if via == "direct":
                prev = O.solve_mh_direct(P)
            else:
                S, r = O.schur2(P)
                prev = O.resolve(P, spla.spsolve(S.tocsc(), r))
            if step % 10 == 0:
                ref = z["ref_pressure_steps"][step // 10]
                p = prev[P.n_sides:P.n_sides + P.n_el]
                assert np.abs(p - ref).max() <= 1e-9 * np.abs(ref).max()
                assert np.abs(zm["ref_pressure_steps"][step // 10] - ref).max() > 1e-3 * np.abs(ref).max()


def z_dt():
    z, _ = load_fixture("t10_mh")
    return z["dt"]


def test_local_matrix_inverse_and_symmetry():
    z, mesh = load_fixture("t01")
    for e in (0, 10, 100, 500, 830):
        A, Ai, det, rc = O.local_matrix(mesh, e, conductivity=2.0, cross_section=0.5)
        assert rc == 0
        n = A.shape[0]
        assert np.allclose(A, A.T, rtol=1e-14, atol=0)
        assert np.allclose(A @ Ai, np.eye(n), atol=1e-12)
        assert np.all(np.linalg.eigvalsh(A) > 0)


def test_cpu_ilu0_pcg():
    """The ILU(0)-preconditioned CG of the CPU baseline: L U equals the edge system on its
    pattern, and the solve reaches the direct solution in fewer iterations than Jacobi."""
    z, mesh, topo, P = problem("t01")
    S, r = O.schur2(P)
    S = S.tocsr()
    S.sort_indices()
    L, U = O.ilu0(S)
    mask = S.copy()
    mask.data[:] = 1.0
    assert abs((L @ U - S).multiply(mask)).max() <= 1e-14 * abs(S).max()
    x, it, res, t_factor = O.pcg_ilu0(S, r, rtol=1e-12)
    _, it_j, _ = O.pcg_jacobi(S, r, rtol=1e-12)
    assert 0 < it < it_j and res <= 1e-12 * 1.01 and t_factor >= 0.0
    import scipy.sparse.linalg as spla
    assert np.abs(x - spla.spsolve(S.tocsc(), r)).max() < 1e-9


def test_cpu_pcg_matches_direct():
    z, mesh, topo, P = problem("t01")
    S, r = O.schur2(P)
    x, it, res = O.pcg_jacobi(S, r, rtol=1e-12)
    assert it > 0 and res <= 1e-12 * 1.01
    import scipy.sparse.linalg as spla
    lam = spla.spsolve(S.tocsc(), r)
    assert np.abs(x - lam).max() < 1e-9


def _dense_iluk(A, pattern, k):
    """Level-of-fill ILU(k) on a dense copy, restated independently of orc_iluk.c (Saad,
    algorithm 10.5): levels start at 0 on the pattern of A (inf elsewhere); row i is
    eliminated with every finished row j < i whose entry (i, j) has level <= k, which updates
    all (i, m) and gives them the level min(lev_im, lev_ij + lev_jm + 1); at the end of the
    row, entries above level k are dropped."""
    n = A.shape[0]
    W = A.copy()
    lev = np.where(pattern, 0, np.inf)
    for i in range(n):
        for j in range(i):
            if lev[i, j] > k:
                continue
            W[i, j] /= W[j, j]
            m = np.arange(j + 1, n)
            m = m[lev[j, m] <= k]
            W[i, m] -= W[i, j] * W[j, m]
            lev[i, m] = np.minimum(lev[i, m], lev[i, j] + lev[j, m] + 1)
        drop = lev[i] > k
        lev[i, drop] = np.inf
        W[i, drop] = 0.0
    return W, lev <= k


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_cpu_iluk_matches_dense_restatement(k):
    """ILU(k) of the CPU baseline (the reference's PETSc preconditioner is ILU(3)): pattern and
    factors equal a dense restatement of the level-of-fill rule on a small fractured system."""
    import cases as OC
    P, mesh, coeffs, topo, bc = OC.problem(1, n=3)
    S, r = O.schur2(P)
    F = O.iluk(S, k, raw=True)
    Sc = S.tocoo()
    spat = np.zeros(S.shape, bool)
    spat[Sc.row, Sc.col] = True
    W, pat = _dense_iluk(S.toarray(), spat, k)
    Fd = F.toarray()
    got_pat = np.zeros_like(pat)
    Fc = F.tocoo()
    got_pat[Fc.row, Fc.col] = True
    assert np.array_equal(got_pat, pat)
    assert np.abs(Fd - np.where(pat, W, 0.0)).max() <= 1e-12 * np.abs(W).max()


def test_cpu_iluk_pcg():
    """ILU(0) through orc_iluk equals orc_ilu0; more levels need fewer iterations; enough
    levels give the exact LU, and PCG converges in one iteration."""
    import cases as OC
    P, mesh, coeffs, topo, bc = OC.problem(1, n=6)
    S, r = O.schur2(P)
    L0, U0 = O.ilu0(S)
    Lk, Uk = O.iluk(S, 0)
    assert abs(L0 - Lk).max() == 0.0 and abs(U0 - Uk).max() == 0.0
    its = []
    for k in (0, 1, 3):
        x, it, res, tf, fill = O.pcg_iluk(S, r, k=k, rtol=1e-10)
        assert it > 0 and res <= 1e-10 * 1.01
        its.append(it)
        if k == 0:
            assert fill == 1.0 and it == O.pcg_ilu0(S, r, rtol=1e-10)[1]
    assert its[0] > its[1] > its[2]
    Lf, Uf = O.iluk(S, 10 ** 6)
    A = S.toarray()
    assert np.abs((Lf @ Uf).toarray() - A).max() <= 1e-13 * np.abs(A).max()
    x, it, res, tf, fill = O.pcg_iluk(S, r, k=10 ** 6, rtol=1e-10)
    assert it <= 1
