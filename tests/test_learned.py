"""Learned smoother (MH_SOLVER_FCG_LEARNED) and flexible CG.

CPU: the NumPy restatement of the network (oracle/smoother_nn.py): its backward against
central differences in FP64; the untrained output is w = 1.  GPU: the network's forward
(tensor-core layers) and its parameter gradient (backward kernels) against that restatement;
the smoother-weight gradient (the V-cycle's adjoint) against finite differences of the GPU's
own loss; flexible-CG solves to tolerance; the fallback; and the ablation trained vs untrained
network on a held-out system (iterations and time)."""
import time

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import mhdarcy
import smoother_nn as SN
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case

CONVERGED = (0, _lib.MH_FELL_BACK)


def random_params(seed, out_scale=0.5):
    """Random hidden layers (the library's initial scale) and a random output layer."""
    th = SN.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    th[SN.PARAMS - SN.WIDTH - 1:] = rng.normal(0.0, out_scale, SN.WIDTH + 1).astype(np.float32)
    th[SN.WIDTH * SN.NFEAT:SN.WIDTH * SN.NFEAT + SN.WIDTH] = rng.normal(0.0, 0.1, SN.WIDTH)  # b0
    return th


def small_scaled(n=4, seed=0):
    import cases as OC
    import oracle as O
    P, *_ = OC.problem(1, n=n, seed=seed)
    S, r = O.schur2(P)
    d = 1.0 / np.sqrt(S.diagonal())
    return (sp.diags(d) @ S @ sp.diags(d)).tocsr()


def test_oracle_backward_finite_differences():
    """backward() of the restatement against central differences of its FP64 forward."""
    Sh = small_scaled()
    x, A = SN.features(Sh)
    th = random_params(3).astype(np.float64)
    w, acts = SN.forward(th, x, A, exact=True)
    c = np.random.default_rng(7).normal(size=len(w))
    g = SN.backward(th, x, A, acts, 2 * c * w)
    gmax = np.abs(g).max()
    for idx in np.random.default_rng(1).choice(SN.PARAMS, 40, replace=False):
        e = 1e-6
        tp, tm = th.copy(), th.copy()
        tp[idx] += e
        tm[idx] -= e
        fd = (np.sum(c * SN.forward(tp, x, A, True)[0] ** 2) - np.sum(c * SN.forward(tm, x, A, True)[0] ** 2)) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 * max(abs(g[idx]), 1e-3 * gmax), (idx, fd, g[idx])


def test_oracle_untrained_output_is_one():
    Sh = small_scaled()
    x, A = SN.features(Sh)
    w, _ = SN.forward(SN.init_params(0), x, A)
    assert np.all(w == 1.0)


def assembled(n, seed=5, cfg=1):
    mesh, coeffs = make_case(cfg, seed=seed, n=n)
    s = mhdarcy.MHSystem(mesh)
    bc, _ = dirichlet_x_bc(s.topology(), mesh)
    s.set_coeffs(**coeffs)
    s.set_bc(bc["bc_type"], bc["pressure"])
    s.assemble()
    return s


def scaled_system(s):
    """The Jacobi-scaled edge system S^ = D^-1/2 S D^-1/2 and b^ = D^-1/2 b (edge order)."""
    rp, col, val, rhs = s.schur_system()
    S = sp.csr_matrix((val, col, rp), shape=(s.n_edges, s.n_edges))
    d = 1.0 / np.sqrt(S.diagonal())
    D = sp.diags(d)
    return (D @ S @ D).tocsr(), d * rhs, S, rhs


def oracle_inputs(s):
    """Features and aggregation matrix of the restatement from the GPU's FP32 scaled matrix."""
    Sh, _, _, _ = scaled_system(s)
    S32 = sp.csr_matrix(Sh.astype(np.float32))
    return SN.features(S32)


@pytest.mark.gpu
def test_forward_matches_oracle(gpu):
    """The network's smoother weights on the GPU (tensor-core layers: bf16 operands, fp32 sums)
    against the NumPy forward with the same bf16 roundings."""
    with assembled(6) as s:
        th = random_params(11)
        s.set_learned_weights(th)
        assert np.array_equal(s.learned_weights(), th)
        w = s.learned_smoother()
        x, A = oracle_inputs(s)
        wref, _ = SN.forward(th, x, A)
        assert w.max() - w.min() > 0.05  # a non-trivial network
        assert np.abs(w - wref).max() <= 2e-3, np.abs(w - wref).max()


@pytest.mark.gpu
def test_untrained_network_is_plain_multigrid(gpu):
    """A new handle's network gives w = 1: the learned method's first solve is the plain
    multigrid's (same iterations)."""
    with assembled(8) as s:
        assert np.all(s.learned_smoother() == 1.0)
        a = s.solve(method=_lib.MH_SOLVER_AMG, r_tol=1e-10)
        b = s.solve(method=_lib.MH_SOLVER_FCG_LEARNED, r_tol=1e-10)
        assert a["status"] == 0 and b["status"] == 0 and a["iterations"] == b["iterations"], (a, b)


def pair(s, k=30, seed=0):
    """A solver pair (r, e) of the held-out kind: CG iterate x_k on S^, r = b^ - S^ x_k, e = x* - x_k,
    scaled by 1/|r| (edge order)."""
    Sh, bh, _, _ = scaled_system(s)
    xs = spla.spsolve(Sh.tocsc(), bh)
    it = [0]
    snap = {}

    def keep(xk):
        it[0] += 1
        if it[0] == k:
            snap["x"] = xk.copy()

    spla.cg(Sh, bh, rtol=1e-14, maxiter=k, callback=keep)
    r = bh - Sh @ snap["x"]
    e = xs - snap["x"]
    sc = 1.0 / np.linalg.norm(r)
    return r * sc, e * sc


@pytest.mark.gpu
def test_parameter_gradient_matches_oracle(gpu):
    """The backward kernels: the GPU's parameter gradient equals the restatement's backward
    applied to the GPU's smoother-weight gradient dL/dw (tolerance 2e-2 of each layer's norm:
    bf16 operands, FP32 sums in another order)."""
    with assembled(6) as s:
        th = random_params(7)
        s.set_learned_weights(th)
        r, e = pair(s)
        loss, g = s.learned_grad(r, e)
        loss2, dw, w = s.learned_grad_weights(r, e, refresh=False)
        assert abs(loss - loss2) <= 1e-6 * abs(loss) and np.abs(dw).max() > 0
        x, A = oracle_inputs(s)
        wref, acts = SN.forward(th, x, A)
        assert np.abs(w - wref).max() <= 2e-3
        gref = SN.backward(th, x, A, acts, dw)
        o = 0
        blocks = [SN.WIDTH * SN.NFEAT + SN.WIDTH] + [SN.WIDTH * 2 * SN.WIDTH + SN.WIDTH] * SN.LAYERS + [SN.WIDTH + 1]
        for b in blocks:
            sl = slice(o, o + b)
            err = np.linalg.norm(g[sl] - gref[sl])
            assert err <= 2e-2 * np.linalg.norm(gref[sl]) + 1e-30, (o, err, np.linalg.norm(gref[sl]))
            o += b


@pytest.mark.gpu
def test_smoother_weight_gradient_finite_differences(gpu):
    """The parameter gradient (the V-cycle's adjoint, then the network's backward) against the
    slope of the GPU loss along the gradient's own direction, for the output layer and for the
    hidden layers (the smoothing interval held fixed, as the gradient assumes).  The FP32 cycle
    makes the loss noisy at the 1e-5 level (rounding through the coarse levels), so each slope
    is a quadratic fit over nine points spanning a loss change far above that noise, and the
    single-parameter differences a noise-free function would allow are not used."""
    with assembled(6) as s:
        th = random_params(5)
        s.set_learned_weights(th)
        r, e = pair(s)
        loss, g = s.learned_grad(r, e)
        s.learned_grad_weights(r, e, refresh=True)  # the interval of the base point
        g = g.astype(np.float64)
        out = slice(SN.PARAMS - SN.WIDTH - 1, SN.PARAMS)
        rows = []
        for name, part in (("output", out), ("hidden", slice(0, out.start))):
            v = np.zeros(SN.PARAMS)
            v[part] = g[part]
            gn = np.linalg.norm(v)
            v /= gn
            h = 2e-3 * abs(loss) / gn  # a loss change of about 0.2%
            ts = np.linspace(-h, h, 9)
            ls = []
            for t in ts:
                s.set_learned_weights((th + t * v).astype(np.float32))
                ls.append(s.learned_grad_weights(r, e, refresh=False)[0])
            slope = np.polyfit(ts, ls, 2)[1]
            rows.append((name, slope, gn, h))
        s.set_learned_weights(th)
        print("directional slopes (part, fit, |g|, step):", rows, "loss", loss)
        for name, slope, gn, _ in rows:
            assert abs(slope - gn) <= 0.1 * gn, (name, slope, gn)


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
        if method == _lib.MH_SOLVER_FCG_LEARNED:
            s.set_learned_weights(random_params(9, out_scale=0.3))
        st = s.solve(method=method, r_tol=1e-10, cheb_degree=4)
        assert st["status"] == 0 and st["fell_back"] == 0, st
        lam, S, rhs = check_solution(s, st, 1e-10)
        lam_direct = spla.spsolve(S.tocsc(), rhs)
        s.solve(method=_lib.MH_SOLVER_PCG64, r_tol=1e-10)
        lam64 = s.solution()[s.n_sides + s.n_elements:]
        err64 = np.abs(lam64 - lam_direct).max()
        assert np.abs(lam - lam_direct).max() <= max(20 * err64, 1e-12)


@pytest.mark.gpu
def test_stalled_learned_solve_falls_back(gpu):
    """A learned segment that uses up its inner iterations hands the solve to Chebyshev-Jacobi,
    which finishes it (status MH_FELL_BACK, the residual criterion met)."""
    with assembled(8) as s:
        st = s.solve(method=_lib.MH_SOLVER_FCG_LEARNED, r_tol=1e-10, inner_rtol=1e-12, inner_max_it=2)
        assert st["status"] == _lib.MH_FELL_BACK and st["fell_back"] == 1, st
        check_solution(s, st, 1e-10)


def timed_solves(s, method, reps=5):
    best, it = 1e30, None
    for _ in range(reps):
        s.assemble()
        st = s.solve(method=method, r_tol=1e-10)
        assert st["status"] in CONVERGED, st
        best = min(best, st["ms_solve"])
        it = st["iterations"]
    return it, best


@pytest.mark.gpu
def test_training_ablation(gpu):
    """Train on one system, evaluate on another of the same family (other seed, larger), the
    trained network against the untrained one (w = 1: the plain multigrid).  Training lowers the
    loss on its pairs and the trained method solves the held-out system to tolerance.  What the
    training gains is measured and printed, and the assertion is that it does not lose
    iterations: on these systems the fine smoother's row weights have no leverage (random or
    row-sum weights leave the iteration count unchanged), so the trained network, which moves
    the weights towards a uniform value that the re-estimated smoothing interval cancels, ends
    with the untrained network's iteration count."""
    with assembled(16, seed=21, cfg=5) as s:
        st = s.learned_train(n_pairs=12, epochs=30, lr=2e-3)
        assert st["n_pairs"] >= 8 and st["loss_final"] <= st["loss_initial"], st
        th = s.learned_weights()
    with assembled(32, seed=22, cfg=5) as s:
        it0, ms0 = timed_solves(s, _lib.MH_SOLVER_FCG_LEARNED)  # untrained: w = 1
        s.set_learned_weights(th)
        it1, ms1 = timed_solves(s, _lib.MH_SOLVER_FCG_LEARNED)
        check_solution(s, None, 1e-10)
        print(f"ablation: training loss {st['loss_initial']:.5f} -> {st['loss_final']:.5f}; held-out iterations "
              f"untrained {it0}, trained {it1}; solve ms untrained {ms0:.2f}, trained {ms1:.2f}")
        assert it1 <= it0, (it0, it1, ms0, ms1)
