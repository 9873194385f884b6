"""The multigrid V-cycle's coarse tail as one thread-block cluster launch (k_tail running the
phase list the host compiles from the hierarchy; MH_AMG_TAIL rows) against the same cycle with
one launch per level kernel (the default): the phases keep the per-level kernels' work split
and summation order, so iterations and solutions are bit-identical.  The larger fractured case
has hub rows (more than 96 entries) on the tail's levels, which the tail handles in 256-thread
groups."""
import numpy as np
import pytest

import mhdarcy
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case


def solve_case(cfg, n, seed, tail_rows, monkeypatch, method=_lib.MH_SOLVER_AMG):
    if tail_rows is None:
        monkeypatch.delenv("MH_AMG_TAIL", raising=False)
    else:
        monkeypatch.setenv("MH_AMG_TAIL", str(tail_rows))
    mesh, coeffs = make_case(cfg, seed=seed, n=n)
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        st = s.solve(method=method, r_tol=1e-10)
        tail = s.amg_tail()
        info = s.amg_info()
        long_rows = 0
        for l in range(max(tail["level"], 1), info["levels"]):
            (rp, _, _), _, _ = s.amg_level(l)
            long_rows += int(np.sum(np.diff(rp) > 96))
        return st, s.solution(), tail, info, long_rows


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,n,seed,tail_rows", [(1, 16, 3, 8192), (5, 24, 7, 8192), (5, 48, 7, 60000)])
def test_tail_matches_per_level_launches(gpu, monkeypatch, cfg, n, seed, tail_rows):
    st0, sol0, tail0, info0, _ = solve_case(cfg, n, seed, 0, monkeypatch)
    st1, sol1, tail1, info1, long_rows = solve_case(cfg, n, seed, tail_rows, monkeypatch)
    assert tail0["level"] == 0 and tail1["level"] >= 1 and tail1["cluster"] in (8, 16), (tail0, tail1, info1)
    assert info0 == info1
    assert st0["status"] == 0 and st1["status"] == 0
    assert st0["iterations"] == st1["iterations"] and st0["outer_iterations"] == st1["outer_iterations"]
    assert np.array_equal(sol0, sol1)
    if cfg == 5:
        print("tail from level", tail1["level"], "of", info1["levels"], "rows", info1["rows"], "hub rows", long_rows)
    if n == 48:
        assert long_rows > 0


@pytest.mark.gpu
def test_tail_in_learned_solve(gpu, monkeypatch):
    """The tail also serves the learned method's cycle (weighted fine smoothing above it)."""
    st0, sol0, _, _, _ = solve_case(1, 12, 5, 0, monkeypatch, _lib.MH_SOLVER_FCG_LEARNED)
    st1, sol1, tail1, _, _ = solve_case(1, 12, 5, 8192, monkeypatch, _lib.MH_SOLVER_FCG_LEARNED)
    assert tail1["level"] >= 1
    assert st0["iterations"] == st1["iterations"] and np.array_equal(sol0, sol1)
