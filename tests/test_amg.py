"""Aggregation multigrid preconditioner (MH_SOLVER_AMG): the hierarchy built on the GPU
against scipy (every coarse matrix is the Galerkin product P^T A P of the level above with the
piecewise-constant P of the exported aggregation, weighted on the finest level; aggregates
hold 1..4 rows on the fine level, 1..8 below), and AMG-FCG solves
to tolerance against the direct solve, single and batched."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import mhdarcy
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case

CONVERGED = (0, _lib.MH_FELL_BACK)


def assembled(n, seed=5, cfg=1):
    mesh, coeffs = make_case(cfg, seed=seed, n=n)
    s = mhdarcy.MHSystem(mesh)
    bc, _ = dirichlet_x_bc(s.topology(), mesh)
    s.set_coeffs(**coeffs)
    s.set_bc(bc["bc_type"], bc["pressure"])
    s.assemble()
    return s


def edge_system(s):
    rp, col, val, rhs = s.schur_system()
    return sp.csr_matrix((val, col, rp), shape=(s.n_edges, s.n_edges)), rhs


def check_solution(s, st, r_tol):
    S, rhs = edge_system(s)
    lam = s.solution()[s.n_sides + s.n_elements:]
    res = rhs - S @ lam
    d = np.sqrt(S.diagonal())
    rel_s = np.linalg.norm(res / d) / np.linalg.norm(rhs / d)
    rel_o = np.linalg.norm(res) / np.linalg.norm(rhs)
    assert rel_s <= 1.1 * r_tol and rel_o <= 1.1 * r_tol, (rel_s, rel_o, st)
    return lam, S, rhs


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,n", [(1, 8), (5, 24)])
def test_amg_hierarchy_is_galerkin(gpu, cfg, n):
    """cfg5 (fracture planes, channels) grows hub rows on its coarse levels: those take the
    long-row kernels and the large Galerkin gather buffer."""
    with assembled(n, cfg=cfg) as s:
        st = s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-8)
        assert st["status"] in CONVERGED and st["fell_back"] == 0, st
        info = s.amg_info()
        assert info["levels"] >= 2
        assert all(info["rows"][l + 1] < info["rows"][l] for l in range(info["levels"] - 1)), info
        for l in range(info["levels"] - 1):
            (rp, col, val), agg, wt = s.amg_level(l)
            (rpc, colc, valc), _, _ = s.amg_level(l + 1)
            n, nc = len(rp) - 1, len(rpc) - 1
            A = sp.csr_matrix((val.astype(np.float64), col, rp), shape=(n, n))
            Ac = sp.csr_matrix((valc.astype(np.float64), colc, rpc), shape=(nc, nc))
            assert agg.min() >= -1 and agg.max() == nc - 1
            sizes = np.bincount(agg[agg >= 0], minlength=nc)
            # two pairing passes from the fine level, three from coarser ones
            assert sizes.min() >= 1 and sizes.max() <= (4 if l == 0 else 8), (l, sizes.min(), sizes.max())
            assert np.all(np.diff(rpc) >= 0)
            keep = np.nonzero(agg >= 0)[0]
            P = sp.csr_matrix((wt[keep].astype(np.float64), (keep, agg[keep])), shape=(n, nc))
            G = (P.T @ A @ P).tocsr()
            diff = abs(G - Ac).max()
            assert diff <= 1e-5 * abs(G).max(), (l, diff, abs(G).max())
            # rows left out of the hierarchy have no off-diagonal coupling (or are padding)
            for i in np.nonzero(agg < 0)[0][:200]:
                offd = [v for c, v in zip(col[rp[i]:rp[i + 1]], val[rp[i]:rp[i + 1]]) if c != i]
                assert l > 0 or not offd or np.allclose(offd, 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(6, 5), (12, 7)])
def test_amg_solve_matches_direct(gpu, n, seed):
    with assembled(n, seed=seed) as s:
        st = s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        assert st["status"] == 0 and st["fell_back"] == 0, st
        lam, S, rhs = check_solution(s, st, 1e-10)
        lam_direct = spla.spsolve(S.tocsc(), rhs)
        s.solve(method=_lib.MH_SOLVER_PCG64, r_tol=1e-10)
        lam64 = s.solution()[s.n_sides + s.n_elements:]
        err64 = np.abs(lam64 - lam_direct).max()
        assert np.abs(lam - lam_direct).max() <= max(20 * err64, 1e-12)
        it64 = s.solve(method=_lib.MH_SOLVER_PCG64, r_tol=1e-10)["iterations"]
        assert st["iterations"] < it64, (st["iterations"], it64)


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,n", [(1, 12), (5, 24)])
def test_amg_fp16_fine_values(gpu, monkeypatch, cfg, n):
    """The cycle's FP16 copy of the fine values (the default) changes the preconditioner only:
    both variants reach the tolerance on the FP64 residual, agree with each other, and need
    about the same number of iterations."""
    out = {}
    for half in ("1", "0"):
        monkeypatch.setenv("MH_AMG_HALF", half)
        with assembled(n, cfg=cfg) as s:
            st = s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
            assert st["status"] == 0 and st["fell_back"] == 0, (half, st)
            lam, S, rhs = check_solution(s, st, 1e-10)
            out[half] = (lam, st["iterations"])
            if half == "0":
                lam_direct = spla.spsolve(S.tocsc(), rhs)
                s.solve(method=_lib.MH_SOLVER_PCG64, r_tol=1e-10)
                err64 = np.abs(s.solution()[s.n_sides + s.n_elements:] - lam_direct).max()
    (l1, it1), (l0, it0) = out["1"], out["0"]
    for lam in (l1, l0):
        assert np.abs(lam - lam_direct).max() <= max(20 * err64, 1e-12)
    assert it1 <= it0 + max(2, it0 // 10), (it1, it0)


@pytest.mark.gpu
def test_amg_batch(gpu):
    parts = [make_case(3, seed=300 + i, n=n, corr_len=0.15) for i, n in enumerate((4, 8, 6))]
    with mhdarcy.MHSystem.batch([m for m, _ in parts]) as b:
        coeffs = {k: np.concatenate([c[k] for _, c in parts]) for k in parts[0][1]}
        bc, _ = dirichlet_x_bc(b.topology(), b.mesh)
        b.set_coeffs(**coeffs)
        b.set_bc(bc["bc_type"], bc["pressure"])
        b.assemble()
        st = b.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        assert st["status"] == 0, st
        ist = b.instance_stats()
        assert np.all(ist["status"] == 0) and np.all(ist["rel_residual"] <= 1e-10), ist
        check_solution(b, st, 1e-10)


@pytest.mark.gpu
def test_amg_unsteady_reuses_hierarchy(gpu):
    """Implicit Euler steps at a fixed dt with time-dependent Dirichlet values: the matrix does
    not change, so the AMG hierarchy of the first step is reused (no setup time) and every
    step still matches FP64 PCG stepping of the same problem."""
    mesh, coeffs = make_case(4, seed=9, n=6)
    sols = {}
    for method in (_lib.MH_SOLVER_AMG, _lib.MH_SOLVER_PCG64):
        with mhdarcy.MHSystem(mesh) as s:
            bc, left = dirichlet_x_bc(s.topology(), mesh)
            s.set_coeffs(**coeffs)
            s.set_bc(bc["bc_type"], bc["pressure"])
            s.unsteady_init(0.01, init_pressure=np.zeros(s.n_elements))
            p = bc["pressure"].copy()
            out = []
            for k in range(1, 6):
                p[left] = 1.0 + 0.5 * np.sin(2 * np.pi * 0.01 * k)
                s.set_bc(bc["bc_type"], p)
                st = s.unsteady_step(0.01, method=method, r_tol=1e-11)
                assert st["status"] == 0, st
                if method == _lib.MH_SOLVER_AMG and k > 1:
                    assert st["ms_setup"] == 0.0, st
                out.append(s.solution())
            sols[method] = out
    for a, b in zip(sols[_lib.MH_SOLVER_AMG], sols[_lib.MH_SOLVER_PCG64]):
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()


@pytest.mark.gpu
def test_boundary_values_need_assembly_before_steady_solve(gpu):
    """New boundary values change the right-hand side: a steady solve needs mh_assemble first."""
    with assembled(4) as s:
        bc, _ = dirichlet_x_bc(s.topology(), s.mesh)
        s.set_bc(bc["bc_type"], 2.0 * bc["pressure"])
        with pytest.raises(_lib.MHError) as ei:
            s.solve(method=_lib.MH_SOLVER_AMG)
        assert ei.value.status == _lib.MH_ERR_STATE
        s.assemble()
        assert s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)["status"] == 0
