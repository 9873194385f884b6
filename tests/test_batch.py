"""Batches of independent systems on meshes of uneven size (one launch sequence, per-instance
convergence): the union numbering, and parity of every instance with its solo solve and with
the oracle's direct solve."""
import numpy as np
import pytest

import mhdarcy
import oracle as O
import topology as T
from helpers import oracle_problem
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case

SIZES = [3, 5, 4, 6, 3]


def instances():
    out = []
    for i, n in enumerate(SIZES):
        mesh, coeffs = make_case(3, seed=100 + i, n=n, corr_len=0.2)
        out.append((mesh, coeffs))
    return out


def test_batch_union_topology_and_offsets():
    inst = instances()
    with mhdarcy.MHSystem.batch([m for m, _ in inst]) as b:
        t = b.topology()
        ref = T.build(b.mesh)
        for k in ("el_side_start", "side_edge", "side_bdr", "bdr_edge", "ngh_element", "ngh_edge"):
            assert np.array_equal(t[k], ref[k]), k
        o = b.instance_offsets()
        assert b.n_instances == len(SIZES)
        for i, (m, _) in enumerate(inst):
            with mhdarcy.MHSystem(m) as s:
                assert o["elements"][i + 1] - o["elements"][i] == s.n_elements
                assert o["sides"][i + 1] - o["sides"][i] == s.n_sides
                assert o["edges"][i + 1] - o["edges"][i] == s.n_edges
                assert o["boundaries"][i + 1] - o["boundaries"][i] == s.n_boundaries
        assert b.sizes.n_instances == len(SIZES)


def batch_inputs(b, inst):
    coeffs = {k: np.concatenate([c[k] for _, c in inst]) for k in inst[0][1]}
    bc, _ = dirichlet_x_bc(b.topology(), b.mesh)
    return coeffs, bc


@pytest.mark.gpu
@pytest.mark.parametrize("method", [_lib.MH_SOLVER_PCG64, _lib.MH_SOLVER_IR32])
def test_batch_matches_solo_and_oracle(gpu, method):
    inst = instances()
    with mhdarcy.MHSystem.batch([m for m, _ in inst]) as b:
        coeffs, bc = batch_inputs(b, inst)
        b.set_coeffs(**coeffs)
        b.set_bc(bc["bc_type"], bc["pressure"])
        b.assemble()
        st = b.solve(method=method, r_tol=1e-12)
        assert st["status"] in (0, _lib.MH_FELL_BACK)
        sol = b.solution()
        ist = b.instance_stats()
        assert np.all(ist["status"] == 0) and np.all(ist["rel_residual"] <= 1e-12)
        assert len(set(ist["iterations"].tolist())) > 1          # instances stop on their own
        for i, (m, c) in enumerate(inst):
            q, p, lam = b.instance_solution(sol, i)
            with mhdarcy.MHSystem(m) as s:
                sbc, _ = dirichlet_x_bc(s.topology(), m)
                s.set_coeffs(**c)
                s.set_bc(sbc["bc_type"], sbc["pressure"])
                s.assemble()
                s.solve(method=method, r_tol=1e-12)
                solo = s.solution()
                P = oracle_problem(m, s.topology(), s.n_edges, c, sbc)
            ref = O.solve_mh_direct(P)
            got = np.concatenate([q, p, lam])
            scale = np.abs(ref).max()
            assert np.abs(got - solo).max() <= 1e-7 * scale
            assert np.abs(got - ref).max() <= 1e-7 * scale


@pytest.mark.gpu
def test_autotune_keeps_results(gpu):
    mesh, coeffs = make_case(1, n=8)
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        s.solve(r_tol=1e-12)
        before = s.solution()
        rp0, col0, val0, rhs0 = s.schur_system()
        tune = s.autotune(32)
        assert tune["rows_per_thread"] in (1, 2, 4) and tune["us_per_iter_fp32"] > 0
        assert tune["sell_rows_per_warp"] == 32 * tune["rows_per_thread"]
        assert tune["k1_group"] in (64, 128, 256) and tune["us_assembly"] > 0
        assert tune["amg_fine_passes"] in (2, 3) and tune["ms_amg_solve"] > 0
        st = s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        assert st["status"] == 0
        # the assembly with the chosen element group gives the same system bit for bit
        s.assemble()
        rp1, col1, val1, rhs1 = s.schur_system()
        assert np.array_equal(val0, val1) and np.array_equal(rhs0, rhs1)
        st = s.solve(r_tol=1e-12)
        assert st["status"] == 0
        after = s.solution()
        assert np.abs(after - before).max() <= 1e-8 * np.abs(before).max()


@pytest.mark.gpu
@pytest.mark.parametrize("method", [_lib.MH_SOLVER_PCG64, _lib.MH_SOLVER_IR32, _lib.MH_SOLVER_AMG,
                                    _lib.MH_SOLVER_CHEB])
def test_device_loop_matches_host_loop(gpu, method):
    """Each Krylov run as one graph launch with a device-side conditional loop (the default)
    gives the host-polled run's per-instance iterations and bit-identical solutions: the loop
    stops when every instance is done, and iterations launched after that are no-ops."""
    inst = instances()
    with mhdarcy.MHSystem.batch([m for m, _ in inst]) as b:
        coeffs, bc = batch_inputs(b, inst)
        b.set_coeffs(**coeffs)
        b.set_bc(bc["bc_type"], bc["pressure"])
        b.assemble()
        out = []
        for host_loop in (False, True, False):
            st = b.solve(method=method, r_tol=1e-10, host_loop=host_loop)
            assert st["status"] in (0, _lib.MH_FELL_BACK), st
            ist = b.instance_stats()
            out.append((st["iterations"], ist["iterations"].copy(), b.solution()))
        for it, per, sol in out[1:]:
            assert it == out[0][0] and np.array_equal(per, out[0][1])
            assert np.array_equal(sol, out[0][2])
