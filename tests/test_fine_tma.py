"""The multigrid's fine-level cycle kernels with the matrix streamed through shared memory by
TMA bulk copies (k_fine_tma, MH_AMG_TMA=1, rings of 2 and 4 stages) against the per-thread
kernels that load it directly (the default): the same row arithmetic in the same order, so
iterations and solutions are bit-identical, for the plain multigrid, a batch of uneven
instances, and the learned method (weighted fine smoothing)."""
import numpy as np
import pytest

import mhdarcy
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case


def solve(mesh, coeffs, tma, monkeypatch, method=_lib.MH_SOLVER_AMG, weights=None):
    monkeypatch.setenv("MH_AMG_TMA", "1" if tma else "0")
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        if weights is not None:
            s.set_learned_weights(weights)
        st = s.solve(method=method, r_tol=1e-10)
        return st, s.solution()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,n,seed,stages", [(1, 16, 3, 4), (5, 24, 7, 4), (2, 24, 1, 2)])
def test_fine_tma_matches_direct_loads(gpu, monkeypatch, cfg, n, seed, stages):
    monkeypatch.setenv("MH_AMG_TMA_STAGES", str(stages))
    mesh, coeffs = make_case(cfg, seed=seed, n=n)
    st0, sol0 = solve(mesh, coeffs, False, monkeypatch)
    st1, sol1 = solve(mesh, coeffs, True, monkeypatch)
    assert st0["status"] == 0 and st1["status"] == 0
    assert st0["iterations"] == st1["iterations"] and np.array_equal(sol0, sol1)


@pytest.mark.gpu
def test_fine_tma_batch_and_learned(gpu, monkeypatch):
    parts = [make_case(3, seed=200 + i, n=n, corr_len=0.2) for i, n in enumerate([3, 6, 4, 8])]
    out = []
    for tma in (False, True):
        monkeypatch.setenv("MH_AMG_TMA", "1" if tma else "0")
        with mhdarcy.MHSystem.batch([m for m, _ in parts]) as b:
            coeffs = {k: np.concatenate([c[k] for _, c in parts]) for k in parts[0][1]}
            bc, _ = dirichlet_x_bc(b.topology(), b.mesh)
            b.set_coeffs(**coeffs)
            b.set_bc(bc["bc_type"], bc["pressure"])
            b.assemble()
            st = b.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
            out.append((st["iterations"], b.instance_stats()["iterations"].copy(), b.solution()))
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    import smoother_nn as SN
    th = SN.init_params(3)
    th[SN.PARAMS - SN.WIDTH - 1:] = np.random.default_rng(4).normal(0.0, 0.3, SN.WIDTH + 1).astype(np.float32)
    mesh, coeffs = make_case(1, seed=5, n=12)
    st0, sol0 = solve(mesh, coeffs, False, monkeypatch, _lib.MH_SOLVER_FCG_LEARNED, th)
    st1, sol1 = solve(mesh, coeffs, True, monkeypatch, _lib.MH_SOLVER_FCG_LEARNED, th)
    assert st0["iterations"] == st1["iterations"] and np.array_equal(sol0, sol1)
