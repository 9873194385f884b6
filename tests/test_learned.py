"""Learned preconditioner and flexible CG.

CPU: the NumPy restatement's gradient against finite differences.  GPU: the inference
(tensor-core) network and the training kernels (loss, gradient) against that restatement;
flexible-CG solves with the Chebyshev-Jacobi and the learned preconditioner to tolerance;
the fallback from a broken network to Chebyshev-Jacobi; and the ablation trained vs
untrained network on the same system."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import learned as NN
import mhdarcy
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case

CONVERGED = (0, _lib.MH_FELL_BACK)


def random_weights(seed, scale=0.2, bias=True):
    rng = np.random.default_rng(seed)
    w = rng.normal(0.0, scale, NN.N_PARAMS).astype(np.float32)
    if not bias:
        for l in range(NN.LAYERS):
            o = l * NN.PER_LAYER
            w[o + NN.H * 2 * NN.K:o + NN.H * 2 * NN.K + NN.H] = 0.0
            w[o + NN.PER_LAYER - NN.K:o + NN.PER_LAYER] = 0.0
    return w


def test_oracle_gradient_finite_differences():
    """loss_and_grad (without bf16 rounding, in FP64) against central differences."""
    n = 48
    rng = np.random.default_rng(0)
    S = sp.diags([-0.45 * np.ones(n - 1), np.ones(n), -0.45 * np.ones(n - 1)], [-1, 0, 1]).tocsr()
    w = random_weights(3, 0.3).astype(np.float64)
    r = rng.normal(size=n)
    e = spla.spsolve(S.tocsc(), r)
    NN.QUANTIZE = False
    try:
        _, g = NN.loss_and_grad(S, r, e, w)
        gmax = np.abs(g).max()
        for idx in rng.choice(NN.N_PARAMS, 60, replace=False):
            h = 1e-6
            wp, wm = w.copy(), w.copy()
            wp[idx] += h
            wm[idx] -= h
            lp, _ = NN.loss_and_grad(S, r, e, wp)
            lm, _ = NN.loss_and_grad(S, r, e, wm)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-5 * max(abs(g[idx]), 0.05 * gmax), (idx, fd, g[idx])
    finally:
        NN.QUANTIZE = True


def assembled(n, seed=5, cfg=1):
    mesh, coeffs = make_case(cfg, seed=seed, n=n)
    s = mhdarcy.MHSystem(mesh)
    bc, _ = dirichlet_x_bc(s.topology(), mesh)
    s.set_coeffs(**coeffs)
    s.set_bc(bc["bc_type"], bc["pressure"])
    s.assemble()
    return s


def scaled_system(s):
    """The Jacobi-scaled edge system S^ = D^-1/2 S D^-1/2 and b^ = D^-1/2 b."""
    rp, col, val, rhs = s.schur_system()
    S = sp.csr_matrix((val, col, rp), shape=(s.n_edges, s.n_edges))
    d = 1.0 / np.sqrt(S.diagonal())
    D = sp.diags(d)
    return (D @ S @ D).tocsr(), d * rhs, S, rhs


@pytest.mark.gpu
@pytest.mark.parametrize("bias", [False, True])
def test_inference_matches_oracle(gpu, bias):
    """Tensor-core inference (bf16 mma, fp32 accumulate) against the NumPy forward."""
    with assembled(4) as s:
        Sh, _, _, _ = scaled_system(s)
        S32 = Sh.astype(np.float32).astype(np.float64)
        w = random_weights(11, bias=bias)
        s.set_learned_weights(w)
        assert np.array_equal(s.learned_weights(), w)
        rng = np.random.default_rng(12)
        r = rng.normal(size=s.n_edges).astype(np.float32).astype(np.float64)
        z = s.learned_apply(r)
        rn = np.sqrt(np.dot(r, r))
        zref, _, _ = NN.forward(S32, (r / rn).astype(np.float32), w)
        zref = zref.astype(np.float64) * rn
        assert np.linalg.norm(z - zref) <= 2e-3 * np.linalg.norm(zref), np.linalg.norm(z - zref) / np.linalg.norm(zref)


@pytest.mark.gpu
def test_identity_network_is_jacobi(gpu):
    """A new handle starts from W2 = b2 = 0: z = r."""
    with assembled(4) as s:
        w = s.learned_weights()
        for l in range(NN.LAYERS):
            o = l * NN.PER_LAYER + NN.H * 2 * NN.K + NN.H
            assert np.all(w[o:o + NN.K * NN.H + NN.K] == 0.0)
        r = np.random.default_rng(1).normal(size=s.n_edges).astype(np.float32).astype(np.float64)
        z = s.learned_apply(r)
        assert np.allclose(z, r, rtol=1e-6, atol=1e-6 * np.abs(r).max())


@pytest.mark.gpu
def test_training_gradient_matches_oracle(gpu):
    """Training forward + backward on the GPU against loss_and_grad (bf16-rounded operands,
    fp32 sums on both sides; tolerance 1e-3 on the loss, 2e-2 on each layer's gradient)."""
    with assembled(4) as s:
        Sh, _, _, _ = scaled_system(s)
        S32 = Sh.astype(np.float32).astype(np.float64)
        w = random_weights(7)
        s.set_learned_weights(w)
        rng = np.random.default_rng(8)
        r = rng.normal(size=s.n_edges).astype(np.float32).astype(np.float64)
        e = spla.spsolve(Sh.tocsc(), r).astype(np.float32).astype(np.float64)
        loss, g = s.learned_grad(r, e)
        L, gref = NN.loss_and_grad(S32, r, e, w)
        assert abs(loss - L) <= 1e-3 * abs(L), (loss, L)
        for l in range(NN.LAYERS):
            sl = slice(l * NN.PER_LAYER, (l + 1) * NN.PER_LAYER)
            err = np.linalg.norm(g[sl] - gref[sl])
            assert err <= 2e-2 * np.linalg.norm(gref[sl]), (l, err, np.linalg.norm(gref[sl]))


def check_solution(s, st, r_tol):
    Sh, bh, S, rhs = scaled_system(s)
    sol = s.solution()
    lam = sol[s.n_sides + s.n_elements:]
    res = rhs - S @ lam
    d = np.sqrt(S.diagonal())
    rel_s = np.linalg.norm(res / d) / np.linalg.norm(rhs / d)
    rel_o = np.linalg.norm(res) / np.linalg.norm(rhs)
    assert rel_s <= 1.1 * r_tol and rel_o <= 1.1 * r_tol, (rel_s, rel_o, st)
    return lam, S, rhs


@pytest.mark.gpu
@pytest.mark.parametrize("method", [_lib.MH_SOLVER_CHEB, _lib.MH_SOLVER_FCG_LEARNED])
def test_fcg_solves_to_tolerance(gpu, method):
    with assembled(8) as s:
        st = s.solve(method=method, r_tol=1e-10, cheb_degree=4)
        assert st["status"] == 0 and st["fell_back"] == 0, st
        lam, S, rhs = check_solution(s, st, 1e-10)
        lam_direct = spla.spsolve(S.tocsc(), rhs)
        s.solve(method=_lib.MH_SOLVER_PCG64, r_tol=1e-10)
        lam64 = s.solution()[s.n_sides + s.n_elements:]
        err64 = np.abs(lam64 - lam_direct).max()
        assert np.abs(lam - lam_direct).max() <= max(20 * err64, 1e-12)


@pytest.mark.gpu
def test_broken_network_falls_back(gpu):
    """Weights whose output overflows to Inf/NaN: the flexible iteration breaks down, the
    solve continues with Chebyshev-Jacobi and still converges (status MH_FELL_BACK)."""
    with assembled(6) as s:
        w = np.full(NN.N_PARAMS, 1e30, np.float32)
        s.set_learned_weights(w)
        st = s.solve(method=_lib.MH_SOLVER_FCG_LEARNED, r_tol=1e-10)
        assert st["status"] == _lib.MH_FELL_BACK and st["fell_back"] == 1, st
        check_solution(s, st, 1e-10)
        assert np.all(s.instance_stats()["status"] == 0)


@pytest.mark.gpu
def test_training_ablation(gpu):
    """Train on one system, evaluate on another of the same family (other seed).  Ablation of
    the training: on the held-out system's own right-hand side the trained network's
    energy-norm error is below the untrained (identity, i.e. Jacobi) network's.  Both networks
    precondition flexible CG to tolerance.  The iteration counts are printed, not compared: the
    trained network is nonlinear in r, which costs flexible CG the conjugacy that the linear
    Jacobi preconditioner keeps, and on these systems it needs more iterations."""
    with assembled(12, seed=21) as s:
        st = s.learned_train(n_pairs=12, epochs=60, lr=2e-3)
        assert st["n_pairs"] >= 8 and st["loss_final"] < 0.95 * st["loss_initial"], st
        w = s.learned_weights()
    with assembled(12, seed=22) as s:
        # held-out pairs made like the training pairs: iterates x_k of CG on S^ (unit diagonal,
        # so Jacobi-PCG), r = b^ - S^ x_k, e = x* - x_k
        Sh, bh, _, _ = scaled_system(s)
        xs = spla.spsolve(Sh.tocsc(), bh)
        snaps = {}
        it = [0]

        def keep(xk):
            it[0] += 1
            if it[0] in (25, 100, 400):
                snaps[it[0]] = xk.copy()

        spla.cg(Sh, bh, rtol=1e-14, maxiter=400, callback=keep)
        pairs = []
        for k in sorted(snaps):
            r = bh - Sh @ snaps[k]
            e = xs - snaps[k]
            sc = 1.0 / np.linalg.norm(r)
            pairs.append(((r * sc).astype(np.float32).astype(np.float64), (e * sc).astype(np.float32).astype(np.float64)))
        assert len(pairs) == 3
        loss_id = np.mean([s.learned_grad(r, e)[0] for r, e in pairs])
        base = s.solve(method=_lib.MH_SOLVER_FCG_LEARNED, r_tol=1e-10)
        assert base["status"] == 0, base
        check_solution(s, base, 1e-10)
        s.set_learned_weights(w)
        loss_tr = np.mean([s.learned_grad(r, e)[0] for r, e in pairs])
        tr = s.solve(method=_lib.MH_SOLVER_FCG_LEARNED, r_tol=1e-10)
        assert tr["status"] in CONVERGED, tr
        check_solution(s, tr, 1e-10)
        print(f"ablation: held-out loss identity {loss_id:.4f}, trained {loss_tr:.4f}; FCG iterations "
              f"identity {base['iterations']}, trained {tr['iterations']}")
        assert loss_tr < loss_id, (loss_tr, loss_id)
