"""mh_csr_residual_noalloc: the residual check for callers that cannot allocate device memory
(for example code running after an allocation has failed, or inside a framework whose memory
pool owns the whole device).  It must report the same residual norms as mh_solve reports for
the same iterate, on repeated calls, without allocating anything itself.

The first call in every context is the set-up call (n = 0): it loads the entry point's code
and looks up its scratch array, which may allocate; the calls checked below come after it.

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


def _noalloc(n, rp, col, val, b, x, r, out, stream):
    v = lambda p: C.c_void_p(p)
    return _lib.lib.mh_csr_residual_noalloc(n, v(rp), v(col), v(val), v(b), v(x), v(r), v(out), v(stream))


def _setup_call(stream=None):
    """The first call in a context: n = 0 does the set-up only."""
    assert _lib.lib.mh_csr_residual_noalloc(0, None, None, None, None, None, None, None,
                                            C.c_void_p(stream)) == _lib.MH_OK


def _device_system(torch, rp, col, val, rhs, lam):
    dev = torch.device("cuda", 0)
    t = dict(rp=torch.as_tensor(rp, dtype=torch.int32, device=dev),
             col=torch.as_tensor(col, dtype=torch.int32, device=dev),
             val=torch.as_tensor(val, dtype=torch.float64, device=dev),
             b=torch.as_tensor(rhs, dtype=torch.float64, device=dev),
             x=torch.as_tensor(lam, dtype=torch.float64, device=dev),
             r=torch.empty(len(rhs), dtype=torch.float64, device=dev),
             out=torch.empty(4, dtype=torch.float64, device=dev))
    return t, torch.cuda.current_stream(dev).cuda_stream


def _call(t, stream, n):
    return _noalloc(n, t["rp"].data_ptr(), t["col"].data_ptr(), t["val"].data_ptr(), t["b"].data_ptr(),
                    t["x"].data_ptr(), t["r"].data_ptr(), t["out"].data_ptr(), stream)


# iterates whose residual is far above the rounding level of b - S x, so the two
# computations (scaled space in mh_solve, unscaled CSR here) agree to the tests' 1e-8
@pytest.mark.parametrize("max_it", [40, 200])
def test_noalloc_residual_matches_mh_solve(gpu, max_it):
    torch = pytest.importorskip("torch")
    st, rp, col, val, rhs, lam = _solver_report(max_it)
    n = len(rhs)
    t, stream = _device_system(torch, rp, col, val, rhs, lam)
    _setup_call(stream)
    S = sp.csr_matrix((val, col, rp), shape=(n, n))
    r_ref = rhs - S @ lam
    # the same (unconverged or converged) iterate twice in a row: the shared scratch keeps the
    # previous call's contents, the results must not depend on it
    for _ in range(2):
        t["r"].fill_(np.nan)
        t["out"].fill_(np.nan)
        assert _call(t, stream, n) == _lib.MH_OK
        out = t["out"].cpu().numpy()
        # residual norms: what mh_solve reported for this iterate
        assert st["rel_residual"] > 1e-6
        np.testing.assert_allclose(out[0], st["rel_residual"], rtol=1e-8)
        np.testing.assert_allclose(out[1], st["rel_residual_unscaled"], rtol=1e-8)
        np.testing.assert_allclose(out[2] / out[3], out[1], rtol=1e-14)
        # the residual vector itself, against a host computation
        r = t["r"].cpu().numpy()
        assert np.abs(r - r_ref).max() <= 1e-12 * np.abs(rhs).max()


def test_noalloc_rejects_oversized_and_aliased_arguments(gpu):
    torch = pytest.importorskip("torch")
    _setup_call()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert _noalloc(_lib.MH_NOALLOC_MAX_ROWS + 1, p, p, p, p, p, p, p, 0) == _lib.MH_ERR_INVALID
    assert _noalloc(-1, p, p, p, p, p, p, p, 0) == _lib.MH_ERR_INVALID
    # r overlapping x or b: rejected before anything runs
    rp = torch.zeros(9, dtype=torch.int32, device="cuda")
    q = rp.data_ptr()
    x, b, r, out = p, p + 64, p + 16, p + 96
    assert _noalloc(4, q, q, p, b, x, x, out, 0) == _lib.MH_ERR_INVALID
    assert _noalloc(4, q, q, p, b, x, r, out, 0) == _lib.MH_ERR_INVALID
    assert _noalloc(4, q, q, p, b, x, b + 16, out, 0) == _lib.MH_ERR_INVALID


def test_noalloc_in_a_second_context(gpu):
    """A driver-API context made current by the caller has its own copy of the scratch array at
    another address: the entry point must look it up there (after that context's set-up call)
    and give the same results, and the primary context's calls must still work afterwards."""
    torch = pytest.importorskip("torch")
    st, rp, col, val, rhs, lam = _solver_report(40)
    n = len(rhs)
    t, stream = _device_system(torch, rp, col, val, rhs, lam)
    _setup_call(stream)
    assert _call(t, stream, n) == _lib.MH_OK
    ref_out, ref_r = t["out"].cpu().numpy(), t["r"].cpu().numpy()
    torch.cuda.synchronize()

    cu = C.CDLL("libcuda.so.1")
    dev, ctx = C.c_int(), C.c_void_p()
    assert cu.cuDeviceGet(C.byref(dev), torch.cuda.current_device()) == 0
    assert cu.cuCtxCreate_v2(C.byref(ctx), 0, dev) == 0  # created and made current
    ptrs = []
    try:
        def upload(a):
            a = np.ascontiguousarray(a)
            d = C.c_uint64()
            assert cu.cuMemAlloc_v2(C.byref(d), C.c_size_t(max(a.nbytes, 8))) == 0
            ptrs.append(d)
            assert cu.cuMemcpyHtoD_v2(d, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)) == 0
            return d.value
        d = [upload(np.asarray(rp, np.int32)), upload(np.asarray(col, np.int32)),
             upload(np.asarray(val, np.float64)), upload(np.asarray(rhs, np.float64)),
             upload(np.asarray(lam, np.float64)), upload(np.zeros(n)), upload(np.full(4, np.nan))]
        _setup_call(None)  # first call in this context
        for _ in range(2):
            assert _noalloc(n, *d, 0) == _lib.MH_OK
            out, r = np.empty(4), np.empty(n)
            assert cu.cuMemcpyDtoH_v2(out.ctypes.data_as(C.c_void_p), C.c_uint64(d[6]), C.c_size_t(32)) == 0
            assert cu.cuMemcpyDtoH_v2(r.ctypes.data_as(C.c_void_p), C.c_uint64(d[5]), C.c_size_t(8 * n)) == 0
            np.testing.assert_array_equal(out, ref_out)
            np.testing.assert_array_equal(r, ref_r)
    finally:
        for p in ptrs:
            cu.cuMemFree_v2(p)
        popped = C.c_void_p()
        cu.cuCtxPopCurrent_v2(C.byref(popped))
        cu.cuCtxDestroy_v2(ctx)
    # back in the primary context: its cached address is still the right one
    t["out"].fill_(np.nan)
    assert _call(t, stream, n) == _lib.MH_OK
    np.testing.assert_array_equal(t["out"].cpu().numpy(), ref_out)
