"""The convection matrix of the explicit transport (mh_transport_matrix; ConvectionTransport::
create_transport_matrix_mpi, transport.cc:788-923) against the oracle's literal restatement
(oracle/transport.py): the same CSR pattern and values within 1e-13 of the largest entry, on
t01 (lines, triangles, tetrahedra, with VB couplings) and on a fractured cube with channels
and random porosity.  The oracle itself is checked for mass conservation on CPU."""
import numpy as np
import pytest

import mhdarcy
import oracle as O
import topology as T
import transport as TR
from helpers import fixture_bc, fixture_coeffs, load_fixture, oracle_problem
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case


def test_oracle_conserves_mass():
    """For a conservative flux field every column j satisfies sum_i V_i a_ij = -(outflow of
    element j across boundary sides): what leaves an element enters its neighbours."""
    z, mesh = load_fixture("t01")
    topo = T.build(mesh)
    co = fixture_coeffs(z)
    P = oracle_problem(mesh, topo, topo["n_edges"], co, fixture_bc(z, topo))
    sol = O.solve_mh_direct(P)
    ne = len(z["el_dim"])
    por = np.random.default_rng(3).uniform(0.1, 0.5, ne)
    A, cfl = TR.transport_matrix(mesh, topo, sol, co["cross_section"], por)
    xyz, eln = np.asarray(mesh.nodes), np.asarray(mesh.el_nodes)
    V = np.array([TR.element_measure(xyz, eln[e], z["el_dim"][e]) for e in range(ne)]) * co["cross_section"] * por
    colsum = A.multiply(V[:, None]).sum(axis=0).A1
    ss, sb = topo["el_side_start"], topo["side_bdr"]
    out = np.array([sum(max(sol[s], 0.0) for s in range(ss[j], ss[j + 1]) if sb[s] >= 0) for j in range(ne)])
    assert np.abs(colsum + out).max() <= 1e-13 * np.abs(sol[:ss[-1]]).max()
    assert cfl == 1.0 / np.abs(A.diagonal()).max()


def t13_problem():
    """tests/13_edge_solute_mixing: the boundary objects of the legacy side-based conditions
    get their flow data (Dirichlet pressures) and transport concentration; the others have no
    condition (no flux) and concentration 0."""
    z, mesh = load_fixture("t13")
    topo = T.build(mesh)
    nb = len(topo["bdr_edge"])
    bt, bp, conc = np.zeros(nb, np.int32), np.zeros(nb), np.zeros(nb)
    ss, sb = topo["el_side_start"], topo["side_bdr"]
    for e, s, typ, val, c in zip(z["lbc_element"], z["lbc_side"], z["lbc_type"], z["lbc_value"], z["lbc_conc"]):
        b = sb[ss[e] + s]
        assert b >= 0
        bt[b], bp[b], conc[b] = typ, val, c
    co = fixture_coeffs(z)
    P = oracle_problem(mesh, topo, topo["n_edges"], co, {"bc_type": bt, "pressure": bp})
    return z, mesh, topo, P, conc


def test_t13_reference_transport_run():
    """The reference's own transport run: the flow outputs of test 13 (printed with 6 digits)
    and the concentrations of its explicit transport at all 200 outputs up to t = 100 (three
    CFL-limited steps per 0.5 interval, mixing where the three strips meet), from the oracle's
    convection matrix, boundary inflow term and time steps."""
    z, mesh, topo, P, conc = t13_problem()
    sol = O.solve_mh_direct(P)
    ns, ne = P.n_sides, P.n_el
    assert np.abs(sol[ns:ns + ne] - z["ref_pressure"]).max() < 2e-5
    assert np.abs(O.element_flux(P, sol) - z["ref_flux"]).max() < 2e-6
    A, cfl = TR.transport_matrix(mesh, topo, sol)
    assert TR.step_count(0.5, cfl) == 3
    c = TR.explicit_transport(A, TR.boundary_inflow(mesh, topo, sol, conc), cfl, np.zeros(ne), z["ref_conc_times"])
    assert len(z["ref_conc_times"]) == 201 and z["ref_conc_times"][-1] == 100.0
    assert np.abs(c - z["ref_conc"]).max() < 5e-6
    assert z["ref_conc"][10].min() < 0.7 < z["ref_conc"][10].max()  # a front is inside the domain at t = 5


def test_t14_time_switched_inflow():
    """The reference's tests/14_trans_time_bc: a uniform flow along a strip, the inflow
    concentration switched by four legacy transport files (20 from t = 1, 0 from 3, 40 from 6,
    0 from 7); the concentrations of its VTK output every 1.0 up to t = 10 (16 digits).  A
    step uses the boundary data of its start time: the output at t = 1 is still all zero."""
    z, mesh = load_fixture("t14")
    topo = T.build(mesh)
    nb = len(topo["bdr_edge"])
    bt, bp = np.zeros(nb, np.int32), np.zeros(nb)
    conc = np.zeros((len(z["lbc_conc_times"]), nb))
    ss, sb = topo["el_side_start"], topo["side_bdr"]
    for j, (e, s, typ, val) in enumerate(zip(z["lbc_element"], z["lbc_side"], z["lbc_type"], z["lbc_value"])):
        b = sb[ss[e] + s]
        assert b >= 0
        bt[b], bp[b] = typ, val
        conc[:, b] = z["lbc_conc_steps"][:, j]
    P = oracle_problem(mesh, topo, topo["n_edges"], fixture_coeffs(z), {"bc_type": bt, "pressure": bp})
    sol = O.solve_mh_direct(P)
    ns, ne = P.n_sides, P.n_el
    assert np.abs(sol[ns:ns + ne] - z["ref_pressure"]).max() < 1e-12
    assert np.abs(O.element_flux(P, sol) - z["ref_flux"]).max() < 1e-12
    A, cfl = TR.transport_matrix(mesh, topo, sol)
    switch = [(t, TR.boundary_inflow(mesh, topo, sol, conc[k])) for k, t in enumerate(z["lbc_conc_times"])]
    c = TR.explicit_transport(A, np.zeros(ne), cfl, np.zeros(ne), z["ref_conc_times"], bc_switch=switch)
    assert np.abs(c - z["ref_conc"]).max() < 1e-9
    assert np.all(z["ref_conc"][1] == 0.0) and z["ref_conc"][7].max() > 39.0


def check_against_oracle(s, mesh, sol, cross_section, porosity):
    (rp, col, val), cfl = s.transport_matrix(porosity)
    A, cfl_ref = TR.transport_matrix(mesh, s.topology(), sol, cross_section,
                                     1.0 if porosity is None else porosity)
    A.sort_indices()
    assert np.array_equal(rp, A.indptr) and np.array_equal(col, A.indices)
    assert np.abs(val - A.data).max() <= 1e-13 * np.abs(A.data).max()
    assert abs(cfl - cfl_ref) <= 1e-13 * cfl_ref
    return val, cfl


@pytest.mark.gpu
def test_transport_matrix_t01(gpu):
    z, mesh = load_fixture("t01")
    co = fixture_coeffs(z)
    with mhdarcy.MHSystem(mesh) as s:
        topo = s.topology()
        bc = fixture_bc(z, topo)
        s.set_coeffs(**co)
        s.set_bc(bc["bc_type"], bc.get("pressure"), bc.get("flux"), bc.get("robin_sigma"))
        s.assemble()
        with pytest.raises(mhdarcy.MHError) as ei:  # no solution yet
            s.transport_matrix()
        assert ei.value.status == _lib.MH_ERR_STATE
        s.solve(r_tol=1e-12)
        check_against_oracle(s, mesh, s.solution(), co["cross_section"], None)


@pytest.mark.gpu
def test_transport_matrix_fractured_cube(gpu):
    torch = pytest.importorskip("torch")
    mesh, coeffs = make_case(5, n=8)
    por = np.random.default_rng(5).uniform(0.05, 0.4, mesh.n_elements)
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        val, cfl = check_against_oracle(s, mesh, s.solution(), coeffs["cross_section"], por)
        # the device variant writes the same values
        buf = torch.full((len(val),), np.nan, dtype=torch.float64, device="cuda:0")
        dpor = torch.as_tensor(por, dtype=torch.float64, device="cuda:0")
        import ctypes as C
        c2 = C.c_double()
        _lib.check(_lib.lib.mh_transport_matrix_device(s.h, dpor.data_ptr(), buf.data_ptr(), buf.numel(),
                                                       C.byref(c2)), s.h)
        assert np.array_equal(buf.cpu().numpy(), val) and c2.value == cfl
