"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference's golden
outputs.

Tolerances:
  * assembled edge system (K1) vs the oracle's element-local double Schur: normwise
    |S_gpu - S_orc|_ij <= 1e-14 sqrt(S_ii S_jj), rhs likewise (identical FP64 element
    arithmetic; only the summation order of the per-entry element contributions differs);
  * back-substitution (K4) given the same edge pressures: 1e-12 relative;
  * solves: the FP64 true residual recomputed by the oracle on its own S2 satisfies the
    criterion (Jacobi-scaled and unscaled relative residual <= 1e-10, with 10% slack for the
    different summation order), and the solution agrees with the FP64 direct solve within
    what that residual allows (checked against the oracle's own Jacobi-PCG at the same
    tolerance); golden fixtures agree with the reference's outputs at the reference's accuracy.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import mhdarcy
import oracle as O
from helpers import cube_bc, fixture_bc, fixture_coeffs, load_fixture, oracle_problem
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case

pytestmark = pytest.mark.gpu

FIXTURES = ["t01", "t05_dirichlet", "t05_neumann", "t05_robin", "t06_32", "t06_21", "t08"]


def gpu_system(mesh, coeffs, bc):
    s = mhdarcy.MHSystem(mesh)
    s.set_coeffs(**coeffs)
    s.set_bc(bc["bc_type"], bc.get("pressure"), bc.get("flux"), bc.get("robin_sigma"))
    s.assemble()
    return s


def fixture_case(name):
    z, mesh = load_fixture(name)
    s = mhdarcy.MHSystem(mesh)
    topo = s.topology()
    coeffs = fixture_coeffs(z)
    bc = fixture_bc(z, topo)
    s.close()
    return z, mesh, coeffs, bc


def scaled_residuals(S, r, lam):
    d = S.diagonal()
    res = r - S @ lam
    rel_s = np.sqrt(np.sum(res ** 2 / d) / np.sum(r ** 2 / d))
    rel_o = np.linalg.norm(res) / np.linalg.norm(r)
    return rel_s, rel_o


def assert_schur_parity(s, P):
    rp, col, val, rhs = s.schur_system()
    S, r = O.schur2(P)
    import scipy.sparse as sp
    G = sp.csr_matrix((val, col, rp), shape=S.shape)
    d = np.sqrt(np.abs(S.diagonal()))
    D = sp.diags(1.0 / d)
    diff = D @ (G - S) @ D
    # the element arithmetic is the oracle's operation for operation (no FMA contraction on
    # either side); only the order in which two or three element contributions are summed
    # into one entry differs
    assert abs(diff).max() <= 1e-14, abs(diff).max()
    # rhs in the same (Jacobi-scaled) units
    assert np.abs((rhs - r) / d).max() <= 1e-14 * np.abs(r / d).max(), np.abs((rhs - r) / d).max()
    return S, r


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_schur_system(gpu, name):
    z, mesh, coeffs, bc = fixture_case(name)
    with gpu_system(mesh, coeffs, bc) as s:
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        assert_schur_parity(s, P)


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("method", [_lib.MH_SOLVER_PCG64, _lib.MH_SOLVER_IR32])
def test_fixture_solution(gpu, name, method):
    z, mesh, coeffs, bc = fixture_case(name)
    with gpu_system(mesh, coeffs, bc) as s:
        st = s.solve(method=method, r_tol=1e-10)
        assert st["status"] in (0, _lib.MH_FELL_BACK) and st["rel_residual"] <= 1e-10
        sol = s.solution()
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        ref = O.solve_mh_direct(P)
        ns, ne = s.n_sides, s.n_elements
        scale = np.abs(ref).max()
        assert np.abs(sol - ref).max() <= 1e-8 * scale
        # the reference's own outputs
        p = sol[ns:ns + ne]
        if "ref_pressure" in z and name == "t01":
            assert np.abs(p - z["ref_pressure"]).max() < 1e-8
        elif "ref_pressure" in z:
            assert np.abs(p - z["ref_pressure"]).max() < 1e-6


def test_t01_side_values_match_raw_output(gpu):
    z, mesh, coeffs, bc = fixture_case("t01")
    with gpu_system(mesh, coeffs, bc) as s:
        s.solve()
        dh = mhdarcy.MH_DofHandler(s, s.solution())
        for e in range(0, s.n_elements, 7):
            n = z["el_dim"][e] + 1
            for i in range(n):
                assert abs(dh.side_scalar(e, i) - z["ref_side_pressure"][e, i]) < 1e-8 + 5e-9 * abs(z["ref_side_pressure"][e, i])
                assert abs(dh.side_flux(e, i) - z["ref_side_flux"][e, i]) < 1e-8 + 5e-9 * abs(z["ref_side_flux"][e, i])
            assert abs(dh.element_scalar(e) - z["ref_pressure"][e]) < 1e-8 + 5e-9 * abs(z["ref_pressure"][e])


def cube(n=8, seed=7, aniso=False, lines=True):
    mesh, coeffs = make_case(1, seed=seed, n=n)
    if not lines:
        mesh, coeffs = make_case(3, seed=seed, n=n)
    if aniso:
        rng = np.random.default_rng(seed)
        ne = mesh.n_elements
        Q = rng.normal(size=(ne, 3, 3))
        A = Q @ np.transpose(Q, (0, 2, 1)) + 3 * np.eye(3)
        coeffs["anisotropy"] = A.reshape(ne, 9)
    s = mhdarcy.MHSystem(mesh)
    bc = cube_bc(s, mesh)
    s.close()
    return mesh, coeffs, bc


@pytest.mark.parametrize("aniso", [False, True])
def test_cube_schur_system(gpu, aniso):
    mesh, coeffs, bc = cube(8, aniso=aniso)
    with gpu_system(mesh, coeffs, bc) as s:
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        assert_schur_parity(s, P)


def test_cube_solve_and_backsub(gpu):
    """cfg1 shape (n=16, fracture + channel, log10 K ~ N(-6,1))."""
    mesh, coeffs = make_case(1)
    with mhdarcy.MHSystem(mesh) as s:
        bc = cube_bc(s, mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        S, r = assert_schur_parity(s, P)
        lam_direct = spla.spsolve(S.tocsc(), r)
        x_cpu, it_cpu, res_cpu = O.pcg_jacobi(S, r, rtol=1e-10)
        err_cpu = np.abs(x_cpu - lam_direct).max()
        for method in (_lib.MH_SOLVER_PCG64, _lib.MH_SOLVER_IR32):
            st = s.solve(method=method, r_tol=1e-10)
            assert st["status"] in (0, _lib.MH_FELL_BACK), st
            sol = s.solution()
            ns, ne = s.n_sides, s.n_elements
            lam = sol[ns + ne:]
            rel_s, rel_o = scaled_residuals(S, r, lam)
            assert rel_s <= 1.1e-10 and rel_o <= 1.1e-10, (rel_s, rel_o)
            assert np.abs(lam - lam_direct).max() <= max(20 * err_cpu, 1e-12), (np.abs(lam - lam_direct).max(), err_cpu)
            # back-substitution parity for the same edge pressures
            ref = O.resolve(P, lam)
            assert np.abs(sol[:ns] - ref[:ns]).max() <= 1e-12 * np.abs(ref[:ns]).max() + 1e-300
            assert np.abs(sol[ns:ns + ne] - ref[ns:ns + ne]).max() <= 1e-12 * np.abs(ref[ns:ns + ne]).max()


def test_tight_tolerance_matches_direct(gpu):
    mesh, coeffs, bc = cube(8)
    with gpu_system(mesh, coeffs, bc) as s:
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        ref, S, r = O.solve_schur_direct(P)
        st = s.solve(r_tol=1e-14)
        assert st["status"] == 0
        sol = s.solution()
        assert np.abs(sol - ref).max() <= 1e-8 * np.abs(ref).max()


def test_element_flux_vectors_t01(gpu):
    """make_element_vector on the device for t01 (lines, triangles, tetrahedra): against the
    oracle on the GPU's own solution (same side fluxes: 1e-12 of the largest vector), and
    against the flux columns of the reference's raw output (printed %.8g)."""
    z, mesh, coeffs, bc = fixture_case("t01")
    with gpu_system(mesh, coeffs, bc) as s:
        with pytest.raises(mhdarcy.MHError) as ei:  # no solution yet
            s.element_flux()
        assert ei.value.status == _lib.MH_ERR_STATE
        s.solve(r_tol=1e-12)
        sol = s.solution()
        u = s.element_flux()
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        ref = O.element_flux(P, sol)
        assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()
        assert np.all(np.abs(u - z["ref_flux"]) <= 1e-8 + 5e-9 * np.abs(z["ref_flux"]))


def test_element_flux_vectors_device_output(gpu):
    """The device-pointer variant writes the same values, on a fractured cube with channels
    and log-normal conductivity and cross-sections (all three element shapes)."""
    torch = pytest.importorskip("torch")
    mesh, coeffs = make_case(5, n=8)
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        sol = s.solution()
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        ref = O.element_flux(P, sol)
        buf = torch.full((s.n_elements, 3), np.nan, dtype=torch.float64, device="cuda:0")
        _lib.check(_lib.lib.mh_get_element_flux_device(s.h, buf.data_ptr(), buf.numel()), s.h)
        u = buf.cpu().numpy()
        assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()
        assert np.array_equal(u, s.element_flux())


def test_node_pressure_and_water_balance_t01(gpu):
    """Node pressures and the water balance of t01 on the device: against the oracle on the
    GPU's own solution, and against the reference's output mesh ($NodeData, %g) and
    water_balance.out (%g)."""
    z, mesh, coeffs, bc = fixture_case("t01")
    with gpu_system(mesh, coeffs, bc) as s:
        with pytest.raises(mhdarcy.MHError) as ei:  # no solution yet
            s.node_pressure()
        assert ei.value.status == _lib.MH_ERR_STATE
        s.solve(r_tol=1e-12)
        sol = s.solution()
        topo = s.topology()
        P = oracle_problem(mesh, topo, s.n_edges, coeffs, bc)
        p = s.node_pressure()
        ref = O.node_pressure(P, sol)
        # one thread per node in the reference's order and operation order: the oracle's bits,
        # and the same bits on every call
        assert np.array_equal(p, ref), np.abs(p - ref).max()
        assert np.array_equal(s.node_pressure(), p)
        rz = z["ref_node_pressure"]
        assert np.all(np.abs(p - rz) <= 5e-6 * np.abs(rz) + 1e-10)
        bids, eids = sorted(set(z["bc_region"].tolist())), sorted(set(z["el_region"].tolist()))
        br = np.array([bids.index(z["bc_region"][b]) for b in topo["bdr_bc_element"]], np.int32)
        er = np.array([eids.index(r) for r in z["el_region"]], np.int32)
        bo, so = s.water_balance(br, er, len(bids), len(eids))
        ob, osrc = O.water_balance(P, sol, br, er)
        scale = np.abs(ob).max()
        assert np.abs(bo - ob).max() <= 1e-12 * scale and np.all(so == 0.0)
        bo2, so2 = s.water_balance(br, er, len(bids), len(eids))
        assert np.array_equal(bo, bo2) and np.array_equal(so, so2)  # deterministic sums
        for rid, *vals in z["ref_bdr_balance"]:
            got = bo[bids.index(int(rid))]
            assert np.all(np.abs(got - vals) <= 5e-6 * np.abs(vals) + 1e-9 * scale), (rid, got, vals)


def test_node_pressure_and_water_balance_sources(gpu):
    """A fractured cube with channels, random cross-sections and water sources, and synthetic
    region maps: node pressures and both balance tables against the oracle; region indices
    out of range are refused."""
    mesh, coeffs = make_case(5, n=8)
    rng = np.random.default_rng(11)
    coeffs = dict(coeffs, water_source_density=rng.normal(0.0, 1e-3, mesh.n_elements))
    with mhdarcy.MHSystem(mesh) as s:
        topo = s.topology()
        bc, _ = dirichlet_x_bc(topo, mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        sol = s.solution()
        P = oracle_problem(mesh, topo, s.n_edges, coeffs, bc)
        ref = O.node_pressure(P, sol)
        assert np.array_equal(s.node_pressure(), ref)
        nb = s.sizes.n_boundaries
        br = (np.arange(nb) % 5).astype(np.int32)
        er = (np.asarray(mesh.el_dim) - 1).astype(np.int32)
        bo, so = s.water_balance(br, er, 5, 3)
        ob, osrc = O.water_balance(P, sol, br, er)
        assert np.abs(bo - ob).max() <= 1e-12 * np.abs(ob).max()
        assert np.abs(so - osrc).max() <= 1e-12 * np.abs(osrc).max() and np.all(osrc != 0.0)
        for _ in range(2):  # deterministic: identical bits on every call
            bo2, so2 = s.water_balance(br, er, 5, 3)
            assert np.array_equal(bo, bo2) and np.array_equal(so, so2)
        with pytest.raises(mhdarcy.MHError) as ei:
            s.water_balance(br, er, 5, 2)  # a tetrahedron has region index 2
        assert ei.value.status == _lib.MH_ERR_INVALID


@pytest.mark.parametrize("cfg", [5, 2])
def test_amg_fluxes_within_1e_8(gpu, cfg):
    """The accuracy target of the mixed-precision multigrid solve: at r_tol 1e-12 the side
    fluxes are within 1e-8 (relative to the largest flux) of the oracle's FP64 direct solution,
    on fractured cases with channels (cfg5 style: six planes, four channels,
    log10 K ~ N(-7, 2)).  Element pressures, whose error the edge residual bounds less tightly,
    within 1e-6 (measured: 2e-8 at n=12, 2e-7 at n=96)."""
    mesh, coeffs = make_case(cfg, n=12)
    s = mhdarcy.MHSystem(mesh)
    try:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc)
        ref, _, _ = O.solve_schur_direct(P)
        st = s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-12)
        assert st["status"] == 0 and st["fell_back"] == 0, st
        sol = s.solution()
        ns, ne = s.n_sides, s.n_elements
        flux_err = np.abs(sol[:ns] - ref[:ns]).max() / np.abs(ref[:ns]).max()
        p_err = np.abs(sol[ns:ns + ne] - ref[ns:ns + ne]).max() / np.abs(ref[ns:ns + ne]).max()
        assert flux_err <= 1e-8 and p_err <= 1e-6, (flux_err, p_err, st["iterations"])
    finally:
        s.close()


def test_unsteady_mh_matches_reference(gpu):
    z, mesh, coeffs, bc = fixture_case("t10_mh")
    dt = float(z["dt"])
    with mhdarcy.MHSystem(mesh) as s:
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.unsteady_init(dt, z["init_pressure"])
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc, time_mode=1, dt=dt)
        prev = np.zeros(s.sizes.mh_size)
        prev[s.n_sides:s.n_sides + s.n_elements] = z["init_pressure"]
        for step in range(1, 51):
            st = s.unsteady_step(dt, r_tol=1e-12)
            assert st["status"] == 0
            sol = s.solution()
            P.set_prev(prev)
            ref = O.solve_mh_direct(P)
            assert np.abs(sol - ref).max() <= 1e-8 * np.abs(ref).max()
            prev = ref
            if step % 10 == 0:
                p = sol[s.n_sides:s.n_sides + s.n_elements]
                r = z["ref_pressure_steps"][step // 10]
                assert np.abs(p - r).max() < 1e-5 * np.abs(r).max()


def test_unsteady_lmh_matches_oracle(gpu):
    z, mesh, coeffs, bc = fixture_case("t10_mh")
    dt = float(z["dt"])
    with mhdarcy.MHSystem(mesh) as s:
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        init = np.linspace(0.0, 1.0, s.n_elements)
        s.unsteady_init(dt, init, lumped=True)
        P = oracle_problem(mesh, s.topology(), s.n_edges, coeffs, bc, time_mode=2, dt=dt)
        prev = np.zeros(s.sizes.mh_size)
        ss, se = s.topology()["el_side_start"], s.topology()["side_edge"]
        for e in range(s.n_elements):
            n = mesh.el_dim[e] + 1
            for i in range(n):
                prev[s.n_sides + s.n_elements + se[ss[e] + i]] += init[e] / n
        for step in range(5):
            st = s.unsteady_step(dt, r_tol=1e-12)
            assert st["status"] == 0
            sol = s.solution()
            P.set_prev(prev)
            S, r = O.schur2(P)
            lam = spla.spsolve(S.tocsc(), r)
            ref = O.resolve(P, lam)
            assert np.abs(sol - ref).max() <= 1e-8 * np.abs(ref).max()
            prev = ref


def test_errors_are_reported(gpu):
    mesh, coeffs, bc = cube(4)
    with mhdarcy.MHSystem(mesh) as s:
        with pytest.raises(mhdarcy.MHError) as ei:
            s.assemble()
        assert ei.value.status == _lib.MH_ERR_STATE
        bad = dict(coeffs)
        bad["conductivity"] = coeffs["conductivity"].copy()
        bad["conductivity"][3] = np.nan
        with pytest.raises(mhdarcy.MHError) as ei:
            s.set_coeffs(**bad)
        assert ei.value.status == _lib.MH_ERR_NONFINITE
        bad["conductivity"][3] = -1.0
        with pytest.raises(mhdarcy.MHError) as ei:
            s.set_coeffs(**bad)
        assert ei.value.status == _lib.MH_ERR_INVALID
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        st = s.solve(max_it=3)
        assert st["status"] == _lib.MH_NOT_CONVERGED
        st = s.solve()
        assert st["status"] == 0


def test_degenerate_element_is_singular(gpu):
    mesh = mhdarcy.cube_mesh(2)
    mesh.nodes[mesh.el_nodes[0, 3]] = mesh.nodes[mesh.el_nodes[0, 0]]  # collapse a tetrahedron
    with mhdarcy.MHSystem(mesh) as s:
        s.set_coeffs(conductivity=np.ones(s.n_elements))
        s.set_bc(np.ones(s.n_boundaries, np.int32), np.zeros(s.n_boundaries))
        with pytest.raises(mhdarcy.MHError) as ei:
            s.assemble()
        assert ei.value.status in (_lib.MH_ERR_SINGULAR, _lib.MH_ERR_NONFINITE)
