"""mh_csr_residual_noalloc: the residual check for callers that cannot allocate device memory
(for example code running after an allocation has failed, or inside a framework whose memory
pool owns the whole device).  It must report the same residual norms as mh_solve reports for
the same iterate, on repeated calls, without allocating anything itself.

This file is named so that pytest collects it last; it passes alone in a fresh process and
after the other tests."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import mhdarcy
from mhdarcy import _lib
from mhdarcy.cases import dirichlet_x_bc, make_case

pytestmark = pytest.mark.gpu


def _solver_report(max_it):
    """An iterate of the edge system and the residual norms mh_solve reports for it."""
    mesh, coeffs = make_case(1, n=8)
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        st = s.solve(max_it=max_it)
        rp, col, val, rhs = s.schur_system()
        lam = s.solution()[s.n_sides + s.n_elements:]
    return st, rp, col, val, rhs, lam


# iterates whose residual is far above the rounding level of b - S x, so the two
# computations (scaled space in mh_solve, unscaled CSR here) agree to the tests' 1e-8
@pytest.mark.parametrize("max_it", [40, 200])
def test_noalloc_residual_matches_mh_solve(gpu, max_it):
    torch = pytest.importorskip("torch")
    st, rp, col, val, rhs, lam = _solver_report(max_it)
    n = len(rhs)
    dev = torch.device("cuda", 0)
    t_rp = torch.as_tensor(rp, dtype=torch.int32, device=dev)
    t_col = torch.as_tensor(col, dtype=torch.int32, device=dev)
    t_val = torch.as_tensor(val, dtype=torch.float64, device=dev)
    t_b = torch.as_tensor(rhs, dtype=torch.float64, device=dev)
    t_x = torch.as_tensor(lam, dtype=torch.float64, device=dev)
    t_r = torch.empty(n, dtype=torch.float64, device=dev)
    t_out = torch.empty(4, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    S = sp.csr_matrix((val, col, rp), shape=(n, n))
    r_ref = rhs - S @ lam
    # the same (unconverged or converged) iterate twice in a row: the shared scratch keeps the
    # previous call's contents, the results must not depend on it
    for _ in range(2):
        t_r.fill_(np.nan)
        t_out.fill_(np.nan)
        rc = _lib.lib.mh_csr_residual_noalloc(n, C.c_void_p(t_rp.data_ptr()), C.c_void_p(t_col.data_ptr()),
                                               C.c_void_p(t_val.data_ptr()), C.c_void_p(t_b.data_ptr()),
                                               C.c_void_p(t_x.data_ptr()), C.c_void_p(t_r.data_ptr()),
                                               C.c_void_p(t_out.data_ptr()), C.c_void_p(stream))
        assert rc == _lib.MH_OK
        out = t_out.cpu().numpy()
        # residual norms: what mh_solve reported for this iterate
        assert st["rel_residual"] > 1e-6
        np.testing.assert_allclose(out[0], st["rel_residual"], rtol=1e-8)
        np.testing.assert_allclose(out[1], st["rel_residual_unscaled"], rtol=1e-8)
        np.testing.assert_allclose(out[2] / out[3], out[1], rtol=1e-14)
        # the residual vector itself, against a host computation
        r = t_r.cpu().numpy()
        assert np.abs(r - r_ref).max() <= 1e-12 * np.abs(rhs).max()


def test_noalloc_rejects_oversized_systems(gpu):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = _lib.lib.mh_csr_residual_noalloc(_lib.MH_NOALLOC_MAX_ROWS + 1, p, p, p, p, p, p, p, None)
    assert rc == _lib.MH_ERR_INVALID
