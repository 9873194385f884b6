"""TEST INFRASTRUCTURE ONLY: Python harness around the C oracle (mh_oracle.c) and scipy.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker of the
GPU library; never imported by the product.  Provides:
  * assemble_mh      -- the full MH saddle-point matrix [sides | elements | edges] as
                        assembly_steady_mh_matrix builds it (src/flow/darcy_flow_mh.cc:525-694);
  * solve_mh_direct  -- FP64 sparse direct solve of that full system (scipy SuperLU): the
                        "FP64 direct oracle", independent of any Schur algebra;
  * schur2 / resolve -- the element-local double Schur complement and back-substitution
                        (src/la/schur.cc:566-773, darcy_flow_mh.cc:1009-1131);
  * pcg_jacobi       -- the CPU FP64 Jacobi-PCG used as the timed CPU baseline;
  * pcg_ilu0 / ilu0  -- CPU FP64 CG with an ILU(0) preconditioner, the zero-fill member of the
                        incomplete factorisations of the reference's PETSc solver (solve.cc:355-374);
  * pcg_iluk / iluk  -- the same with k levels of fill (orc_iluk.c); k = 3 is the reference's
                        serial default (-pc_factor_levels 3, solve.cc:370).
Parity of the restatement is pinned to the reference's golden outputs in tests/golden.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libmhoracle.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB):
        build()
    L = C.CDLL(_LIB)
    i32p, f64p = C.POINTER(C.c_int32), C.POINTER(C.c_double)
    L.orc_assemble_mh.restype = C.c_int64
    L.orc_assemble_mh.argtypes = [C.c_void_p, i32p, i32p, f64p, C.c_int64, f64p]
    L.orc_schur2_coo.restype = C.c_int64
    L.orc_schur2_coo.argtypes = [C.c_void_p, i32p, i32p, f64p, C.c_int64, f64p]
    L.orc_schur2_csr.restype = C.c_int
    L.orc_schur2_csr.argtypes = [C.c_void_p, i32p, i32p, f64p, f64p]
    L.orc_resolve.restype = C.c_int
    L.orc_resolve.argtypes = [C.c_void_p, f64p]
    L.orc_element_flux.restype = C.c_int
    L.orc_element_flux.argtypes = [C.c_void_p, f64p, f64p]
    L.orc_node_pressure.restype = C.c_int
    L.orc_node_pressure.argtypes = [C.c_void_p, f64p, f64p]
    L.orc_water_balance.restype = C.c_int
    L.orc_water_balance.argtypes = [C.c_void_p, f64p, i32p, C.c_int32, i32p, C.c_int32, f64p, f64p]
    L.orc_pcg_jacobi.restype = C.c_int
    L.orc_pcg_jacobi.argtypes = [C.c_int64, i32p, i32p, f64p, f64p, f64p, C.c_double, C.c_int, f64p]
    L.orc_pcg_ilu0.restype = C.c_int
    L.orc_pcg_ilu0.argtypes = [C.c_int64, i32p, i32p, f64p, f64p, f64p, C.c_double, C.c_int, f64p, f64p]
    L.orc_ilu0.restype = C.c_int
    L.orc_ilu0.argtypes = [C.c_int64, i32p, i32p, f64p, f64p, i32p]
    L.orc_local_matrix.restype = C.c_int
    L.orc_local_matrix.argtypes = [f64p, i32p, i32p, C.c_int64, f64p, C.c_double, C.c_double, f64p, f64p, f64p]
    L.orc_num_threads.restype = C.c_int
    L.orc_set_threads.restype = None
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_topology.restype = C.c_int
    L.orc_topology.argtypes = [C.c_int64, C.c_int64, i32p, i32p, C.c_int64, i32p, i32p] + [i32p] * 8 + \
        [C.POINTER(C.c_int64)]
    L.orc_iluk.restype = C.c_int64
    L.orc_iluk.argtypes = [C.c_int64, i32p, i32p, f64p, C.c_int, i32p, i32p, f64p, i32p, C.c_int64]
    L.orc_pcg_iluk.restype = C.c_int
    L.orc_pcg_iluk.argtypes = [C.c_int64, i32p, i32p, f64p, f64p, f64p, C.c_int, C.c_double, C.c_int, f64p, f64p,
                               f64p]
    return L


lib = _load()


class _Problem(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("xyz", C.c_void_p), ("n_el", C.c_int64),
                ("el_dim", C.c_void_p), ("el_nodes", C.c_void_p),
                ("el_side_start", C.c_void_p), ("side_edge", C.c_void_p), ("side_bdr", C.c_void_p),
                ("n_edges", C.c_int64), ("n_ngh", C.c_int64),
                ("ngh_element", C.c_void_p), ("ngh_edge", C.c_void_p), ("ngh_side", C.c_void_p),
                ("K", C.c_void_p), ("aniso", C.c_void_p), ("delta", C.c_void_p), ("sigma", C.c_void_p),
                ("source", C.c_void_p), ("storativity", C.c_void_p),
                ("bc_type", C.c_void_p), ("bc_p", C.c_void_p), ("bc_flux", C.c_void_p),
                ("bc_sigma", C.c_void_p), ("time_mode", C.c_int32), ("dt", C.c_double),
                ("prev", C.c_void_p)]


def _p(a):
    return None if a is None else a.ctypes.data


class Problem:
    """Mesh + topology + coefficients + boundary data, as flat arrays."""

    def __init__(self, mesh, topo, n_edges, conductivity=1.0, anisotropy=None, cross_section=1.0,
                 sigma=1.0, water_source_density=0.0, storativity=1.0, bc_type=0, bc_pressure=0.0,
                 bc_flux=0.0, bc_robin_sigma=0.0, time_mode=0, dt=1.0, prev=None):
        ne = len(mesh.el_dim)
        nb = len(topo["bdr_edge"])
        f = lambda v, n: np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float64), (n,)).copy())
        self.keep = dict(
            xyz=np.ascontiguousarray(mesh.nodes, np.float64), el_dim=np.ascontiguousarray(mesh.el_dim, np.int32),
            el_nodes=np.ascontiguousarray(mesh.el_nodes, np.int32),
            el_side_start=np.ascontiguousarray(topo["el_side_start"], np.int32),
            side_edge=np.ascontiguousarray(topo["side_edge"], np.int32),
            side_bdr=np.ascontiguousarray(topo["side_bdr"], np.int32),
            ngh_element=np.ascontiguousarray(topo["ngh_element"], np.int32),
            ngh_edge=np.ascontiguousarray(topo["ngh_edge"], np.int32),
            ngh_side=np.ascontiguousarray(topo["ngh_side"], np.int32),
            K=f(conductivity, ne), delta=f(cross_section, ne), sigma=f(sigma, ne),
            source=f(water_source_density, ne), storativity=f(storativity, ne),
            aniso=None if anisotropy is None else np.ascontiguousarray(np.asarray(anisotropy, np.float64).reshape(ne, 9)),
            bc_type=np.ascontiguousarray(np.broadcast_to(np.asarray(bc_type, np.int32), (nb,)).copy()),
            bc_p=f(bc_pressure, nb), bc_flux=f(bc_flux, nb), bc_sigma=f(bc_robin_sigma, nb))
        self.n_el = ne
        self.n_sides = int(topo["el_side_start"][-1])
        self.n_edges = n_edges
        self.mh_size = self.n_sides + ne + n_edges
        self.time_mode = time_mode
        self.dt = dt
        self.set_prev(prev)

    def set_prev(self, prev):
        self.keep["prev"] = None if prev is None else np.ascontiguousarray(prev, np.float64)

    def struct(self):
        k = self.keep
        return _Problem(len(k["xyz"]), _p(k["xyz"]), self.n_el, _p(k["el_dim"]), _p(k["el_nodes"]),
                        _p(k["el_side_start"]), _p(k["side_edge"]), _p(k["side_bdr"]), self.n_edges,
                        len(k["ngh_element"]), _p(k["ngh_element"]), _p(k["ngh_edge"]), _p(k["ngh_side"]),
                        _p(k["K"]), _p(k["aniso"]), _p(k["delta"]), _p(k["sigma"]), _p(k["source"]),
                        _p(k["storativity"]), _p(k["bc_type"]), _p(k["bc_p"]), _p(k["bc_flux"]),
                        _p(k["bc_sigma"]), self.time_mode, self.dt, _p(k["prev"]))


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def assemble_mh(P):
    """Full MH matrix (CSR, duplicates summed) and rhs."""
    cap = 64 * P.n_el + 16
    I = np.zeros(cap, np.int32)
    J = np.zeros(cap, np.int32)
    V = np.zeros(cap)
    rhs = np.zeros(P.mh_size)
    s = P.struct()
    k = lib.orc_assemble_mh(C.byref(s), _ptr(I, C.c_int32), _ptr(J, C.c_int32), _ptr(V, C.c_double), cap,
                            _ptr(rhs, C.c_double))
    if k < 0:
        raise RuntimeError(f"orc_assemble_mh failed ({k})")
    A = sp.coo_matrix((V[:k], (I[:k], J[:k])), shape=(P.mh_size, P.mh_size)).tocsr()
    A.sum_duplicates()
    return A, rhs


def solve_mh_direct(P):
    """FP64 direct solve of the full saddle-point MH system."""
    A, rhs = assemble_mh(P)
    return spla.spsolve(A.tocsc(), rhs)


def _local_sizes(P):
    """Edges of each element's local system: its sides plus its VB neighbours' higher sides."""
    m = P.keep["el_dim"].astype(np.int64) + 1
    if len(P.keep["ngh_element"]):
        m += np.bincount(P.keep["ngh_element"], minlength=P.n_el)
    return m


def schur2(P):
    """Second Schur complement S2 (reference schur2 after scale(-1)) and its rhs."""
    cap = int(np.sum(_local_sizes(P) ** 2)) + 16
    I = np.zeros(cap, np.int32)
    J = np.zeros(cap, np.int32)
    V = np.zeros(cap)
    rhs = np.zeros(P.n_edges)
    s = P.struct()
    k = lib.orc_schur2_coo(C.byref(s), _ptr(I, C.c_int32), _ptr(J, C.c_int32), _ptr(V, C.c_double), cap,
                           _ptr(rhs, C.c_double))
    if k < 0:
        raise RuntimeError(f"orc_schur2_coo failed ({k})")
    S = sp.coo_matrix((V[:k], (I[:k], J[:k])), shape=(P.n_edges, P.n_edges)).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    return S, rhs


def schur2_element_blocks(P):
    """The element-local blocks of the second Schur complement in element order, as
    SchurComplement would hand them to LinSys::mat_set_values: (rows, vals) per element with
    rows the element's local edges and vals the m x m block; and the summed rhs."""
    m = _local_sizes(P)
    cap = int(np.sum(m ** 2)) + 16
    I = np.zeros(cap, np.int32)
    J = np.zeros(cap, np.int32)
    V = np.zeros(cap)
    rhs = np.zeros(P.n_edges)
    s = P.struct()
    k = lib.orc_schur2_coo(C.byref(s), _ptr(I, C.c_int32), _ptr(J, C.c_int32), _ptr(V, C.c_double), cap,
                           _ptr(rhs, C.c_double))
    if k != int(np.sum(m ** 2)):
        raise RuntimeError(f"orc_schur2_coo failed ({k})")
    blocks, o = [], 0
    for me in m:
        me = int(me)
        blocks.append((I[o:o + me * me:me].copy(), V[o:o + me * me].reshape(me, me).copy()))
        o += me * me
    return blocks, rhs


def schur2_csr_into(P, row_ptr, col, val, rhs):
    """Fills val/rhs on a given sorted CSR pattern (threaded; the CPU baseline's assembly)."""
    s = P.struct()
    rc = lib.orc_schur2_csr(C.byref(s), _ptr(row_ptr, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double),
                            _ptr(rhs, C.c_double))
    if rc:
        raise RuntimeError("singular local matrix")


def resolve(P, lam):
    """Full MH solution from the edge pressures."""
    sol = np.zeros(P.mh_size)
    sol[P.n_sides + P.n_el:] = lam
    s = P.struct()
    if lib.orc_resolve(C.byref(s), _ptr(sol, C.c_double)):
        raise RuntimeError("singular local matrix")
    return sol


def element_flux(P, sol):
    """Darcy flux vector at every element centre from the side fluxes of an MH solution
    (DarcyFlowMHOutput::make_element_vector, darcy_flow_mh_output.cc:301-323): [n_el, 3]."""
    out = np.zeros((P.n_el, 3))
    s = P.struct()
    lib.orc_element_flux(C.byref(s), _ptr(np.ascontiguousarray(sol, np.float64), C.c_double), _ptr(out, C.c_double))
    return out


def node_pressure(P, sol):
    """Pressure at every node, DarcyFlowMHOutput::make_node_scalar_param
    (darcy_flow_mh_output.cc:424-546): [n_nodes]."""
    out = np.zeros(len(P.keep["xyz"]))
    s = P.struct()
    lib.orc_node_pressure(C.byref(s), _ptr(np.ascontiguousarray(sol, np.float64), C.c_double), _ptr(out, C.c_double))
    return out


def water_balance(P, sol, bdr_region, el_region):
    """DarcyFlowMHOutput::water_balance (darcy_flow_mh_output.cc:671-790) for region indices
    bdr_region [n_bdr] and el_region [n_el]: ([n_bdr_regions, 3] total, outflow, inflow;
    [n_el_regions] sources)."""
    br = np.ascontiguousarray(bdr_region, np.int32)
    er = np.ascontiguousarray(el_region, np.int32)
    nb, ne = int(br.max()) + 1 if br.size else 0, int(er.max()) + 1 if er.size else 0
    ob, os_ = np.zeros((nb, 3)), np.zeros(ne)
    s = P.struct()
    lib.orc_water_balance(C.byref(s), _ptr(np.ascontiguousarray(sol, np.float64), C.c_double), _ptr(br, C.c_int32),
                          nb, _ptr(er, C.c_int32), ne, _ptr(ob, C.c_double), _ptr(os_, C.c_double))
    return ob, os_


def solve_schur_direct(P):
    S, r = schur2(P)
    lam = spla.spsolve(S.tocsc(), r)
    return resolve(P, lam), S, r


def pcg_jacobi(S, b, x0=None, rtol=1e-10, max_it=100000):
    """CPU FP64 Jacobi-PCG on CSR (threaded).  Returns x, iterations (-1 if max_it), rel residual."""
    S = S.tocsr()
    rp = np.ascontiguousarray(S.indptr, np.int32)
    col = np.ascontiguousarray(S.indices, np.int32)
    val = np.ascontiguousarray(S.data, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
    res = C.c_double(0.0)
    it = lib.orc_pcg_jacobi(len(b), _ptr(rp, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double),
                            _ptr(b, C.c_double), _ptr(x, C.c_double), rtol, max_it, C.byref(res))
    return x, it, res.value


def pcg_ilu0(S, b, x0=None, rtol=1e-10, max_it=100000):
    """CPU FP64 CG preconditioned by ILU(0) (IC(0) in LU form for the SPD edge system; the
    triangular solves are sequential).  Returns x, iterations (-1 if max_it, -2 if the
    factorisation failed), the true Jacobi-scaled relative residual and the factorisation's
    seconds."""
    S = S.tocsr()
    S.sort_indices()
    rp = np.ascontiguousarray(S.indptr, np.int32)
    col = np.ascontiguousarray(S.indices, np.int32)
    val = np.ascontiguousarray(S.data, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
    res, tf = C.c_double(0.0), C.c_double(0.0)
    it = lib.orc_pcg_ilu0(len(b), _ptr(rp, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double),
                          _ptr(b, C.c_double), _ptr(x, C.c_double), rtol, max_it, C.byref(res), C.byref(tf))
    return x, it, res.value, tf.value


def _csr_arrays(S):
    S = S.tocsr()
    S.sort_indices()
    return (np.ascontiguousarray(S.indptr, np.int32), np.ascontiguousarray(S.indices, np.int32),
            np.ascontiguousarray(S.data, np.float64))


def pcg_iluk(S, b, k=3, x0=None, rtol=1e-10, max_it=100000):
    """CPU FP64 CG preconditioned by ILU(k) (level-of-fill incomplete LU, orc_iluk.c; k = 3 is
    PETSc's setting in the reference's serial solver).  Returns x, iterations (-1 if max_it,
    -2 if the factorisation failed), the true Jacobi-scaled relative residual, the
    factorisation's seconds and the factor's fill ratio nnz(LU) / nnz(S)."""
    rp, col, val = _csr_arrays(S)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
    res, tf, fill = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
    it = lib.orc_pcg_iluk(len(b), _ptr(rp, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double),
                          _ptr(b, C.c_double), _ptr(x, C.c_double), k, rtol, max_it, C.byref(res), C.byref(tf),
                          C.byref(fill))
    return x, it, res.value, tf.value, fill.value


def iluk(S, k, raw=False):
    """(L, U) of ILU(k) as scipy CSR matrices (L unit lower), for checks; raw=True returns the
    factor as stored (strict L and U in one CSR, its pattern kept with any zero values)."""
    rp, col, val = _csr_arrays(S)
    n = S.shape[0]
    frp = np.zeros(n + 1, np.int32)
    dpos = np.zeros(n, np.int32)
    nnz = lib.orc_iluk(n, _ptr(rp, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double), k,
                       _ptr(frp, C.c_int32), None, None, _ptr(dpos, C.c_int32), 0)
    if nnz < 0:
        raise ArithmeticError("ILU(k) breakdown (%d)" % nnz)
    fcol = np.zeros(nnz, np.int32)
    fval = np.zeros(nnz)
    rc = lib.orc_iluk(n, _ptr(rp, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double), k,
                      _ptr(frp, C.c_int32), _ptr(fcol, C.c_int32), _ptr(fval, C.c_double), _ptr(dpos, C.c_int32), nnz)
    if rc < 0:
        raise ArithmeticError("ILU(k) breakdown (%d)" % rc)
    F = sp.csr_matrix((fval, fcol, frp), shape=S.shape)
    if raw:
        return F
    L = sp.tril(F, -1, format="csr") + sp.identity(n, format="csr")
    return L, sp.triu(F, 0, format="csr")


def ilu0(S):
    """(L, U) of ILU(0) as scipy CSR matrices (L unit lower), for checks."""
    S = S.tocsr()
    S.sort_indices()
    rp = np.ascontiguousarray(S.indptr, np.int32)
    col = np.ascontiguousarray(S.indices, np.int32)
    val = np.ascontiguousarray(S.data, np.float64)
    lu = np.empty_like(val)
    dpos = np.empty(S.shape[0], np.int32)
    if lib.orc_ilu0(S.shape[0], _ptr(rp, C.c_int32), _ptr(col, C.c_int32), _ptr(val, C.c_double),
                    _ptr(lu, C.c_double), _ptr(dpos, C.c_int32)):
        raise ArithmeticError("ILU(0) breakdown")
    F = sp.csr_matrix((lu, col, rp), shape=S.shape)
    L = sp.tril(F, -1, format="csr") + sp.identity(S.shape[0], format="csr")
    return L, sp.triu(F, 0, format="csr")


def local_matrix(mesh, e, conductivity=1.0, cross_section=1.0, anisotropy=None):
    A = np.zeros(16)
    Ai = np.zeros(16)
    det = C.c_double(0.0)
    an = None if anisotropy is None else np.ascontiguousarray(anisotropy, np.float64).reshape(9)
    rc = lib.orc_local_matrix(_ptr(np.ascontiguousarray(mesh.nodes), C.c_double),
                              _ptr(np.ascontiguousarray(mesh.el_nodes), C.c_int32),
                              _ptr(np.ascontiguousarray(mesh.el_dim), C.c_int32), e,
                              None if an is None else _ptr(an, C.c_double), conductivity, cross_section,
                              _ptr(A, C.c_double), _ptr(Ai, C.c_double), C.byref(det))
    n = int(mesh.el_dim[e]) + 1
    return A[:n * n].reshape(n, n), Ai[:n * n].reshape(n, n), det.value, rc


def num_threads():
    return lib.orc_num_threads()


def set_threads(n):
    """OpenMP threads of the following oracle calls."""
    lib.orc_set_threads(int(n))
