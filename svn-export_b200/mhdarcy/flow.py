"""Host-side mirror of the reference's DarcyFlowMH interface over the C ABI.

Names follow the reference: DarcyFlowMH_Steady.update_solution / get_solution_vector
(src/flow/darcy_flow_mh.cc:375-433, 485-500), DarcyFlowMH_Unsteady and
DarcyFlowLMH_Unsteady (:1601-1827), and the MH_DofHandler accessors side_flux / side_scalar
/ element_scalar (src/flow/mh_dofhandler.cc:37-50).  All compute runs in libmhdarcy.so on
the GPU; every error is raised, nothing falls back to the CPU.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import lib, check, f64, i32, ptr


def solve_opts(method=_lib.MH_SOLVER_PCG64, r_tol=1e-10, a_tol=0.0, max_it=20000,
               use_initial_guess=False, inner_rtol=0.0, inner_max_it=2000, iters_per_graph=0,
               cheb_degree=4, profile_kernels=False, host_loop=False):
    o = _lib.SolveOpts()
    lib.mh_solve_opts_default(C.byref(o))
    o.method = method
    o.r_tol = r_tol
    o.a_tol = a_tol
    o.max_it = max_it
    o.use_initial_guess = int(bool(use_initial_guess))
    o.inner_rtol = inner_rtol
    o.inner_max_it = inner_max_it
    o.iters_per_graph = iters_per_graph
    o.cheb_degree = cheb_degree
    o.profile_kernels = int(bool(profile_kernels))
    o.host_loop = int(bool(host_loop))
    return o


class MHSystem:
    """One mixed-hybrid Darcy system on the GPU (an mh_handle), or a batch of independent
    systems (see :meth:`batch`) solved together with per-instance convergence."""

    def __init__(self, mesh, _batch=None, mortar=None):
        """mortar: (method, sigma, master, slave, master_t, slave_xy) of mh_create_mortar
        (see mhdarcy.mortar.plane_intersections), or None."""
        self.mesh = mesh
        h = C.c_void_p()
        if _batch is None:
            d = mesh.desc()
            if mortar is None:
                check(lib.mh_create(C.byref(d), C.byref(h)))
            else:
                from .mortar import mortar_desc
                md, keep = mortar_desc(*mortar)
                check(lib.mh_create_mortar(C.byref(d), C.byref(md), C.byref(h)))
            self.n_instances = 1
        else:
            descs = (_lib.MeshDesc * len(_batch))(*[m.desc() for m in _batch])
            check(lib.mh_create_batch(descs, len(_batch), C.byref(h)))
            self.n_instances = len(_batch)
            self._meshes = _batch
        self.h = h
        s = _lib.Sizes()
        check(lib.mh_get_sizes(h, C.byref(s)))
        self.sizes = s
        self._topo = None

    @classmethod
    def batch(cls, meshes):
        """Independent meshes in one handle.  Element, boundary and solution arrays cover the
        union, each part concatenated over the instances in order."""
        from .mesh import concat_meshes
        s = cls(None, _batch=list(meshes))
        s.mesh = concat_meshes(s._meshes)
        return s

    def instance_offsets(self):
        n = self.n_instances + 1
        arrs = [np.zeros(n, np.int64) for _ in range(4)]
        check(lib.mh_get_instance_offsets(self.h, *[a.ctypes.data_as(C.POINTER(C.c_int64)) for a in arrs]),
              self.h)
        return dict(zip(("elements", "sides", "edges", "boundaries"), arrs))

    def instance_stats(self):
        n = self.n_instances
        it = np.zeros(n, np.int32)
        rel = np.zeros(n)
        st = np.zeros(n, np.int32)
        check(lib.mh_get_instance_stats(self.h, ptr(it, C.c_int32), ptr(rel, C.c_double), ptr(st, C.c_int32)),
              self.h)
        return dict(iterations=it, rel_residual=rel, status=st)

    def autotune(self, iterations=64):
        """Times the launch shapes on the assembled system and keeps the fastest: rows per
        thread of the Krylov kernels (SELL-32 rows per warp 32 R) and the element group of
        the assembly's K1 kernel (mh_autotune_ex)."""
        t = _lib.TuneResult()
        check(lib.mh_autotune_ex(self.h, iterations, C.byref(t)), self.h)
        return t.as_dict()

    def instance_solution(self, sol, i):
        """(side fluxes, element pressures, edge pressures) of instance i from a union solution."""
        o = self.instance_offsets()
        ns, ne = self.n_sides, self.n_elements
        return (sol[o["sides"][i]:o["sides"][i + 1]], sol[ns + o["elements"][i]:ns + o["elements"][i + 1]],
                sol[ns + ne + o["edges"][i]:ns + ne + o["edges"][i + 1]])

    def set_stream(self, cuda_stream):
        """Issue all work on the caller's cudaStream_t (an int handle, e.g. torch's
        Stream.cuda_stream); None returns to the handle's own stream."""
        check(lib.mh_set_stream(self.h, C.c_void_p(cuda_stream) if cuda_stream else None), self.h)

    def kernel_launches(self):
        return lib.mh_kernel_launches(self.h)

    def close(self):
        if self.h:
            lib.mh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def n_sides(self):
        return self.sizes.n_sides

    @property
    def n_elements(self):
        return self.sizes.n_elements

    @property
    def n_edges(self):
        return self.sizes.n_edges

    @property
    def n_boundaries(self):
        return self.sizes.n_boundaries

    def topology(self):
        if self._topo is None:
            s = self.sizes
            t = {
                "el_side_start": np.zeros(s.n_elements + 1, np.int32),
                "side_edge": np.zeros(s.n_sides, np.int32),
                "side_bdr": np.zeros(s.n_sides, np.int32),
                "bdr_bc_element": np.zeros(max(s.n_boundaries, 1), np.int32),
                "bdr_edge": np.zeros(max(s.n_boundaries, 1), np.int32),
                "ngh_element": np.zeros(max(s.n_neighbours, 1), np.int32),
                "ngh_edge": np.zeros(max(s.n_neighbours, 1), np.int32),
                "ngh_side": np.zeros(max(s.n_neighbours, 1), np.int32),
            }
            check(lib.mh_get_topology(self.h, *[ptr(t[k], C.c_int32) for k in
                                                ("el_side_start", "side_edge", "side_bdr",
                                                 "bdr_bc_element", "bdr_edge", "ngh_element",
                                                 "ngh_edge", "ngh_side")]), self.h)
            for k, n in (("bdr_bc_element", s.n_boundaries), ("bdr_edge", s.n_boundaries),
                         ("ngh_element", s.n_neighbours), ("ngh_edge", s.n_neighbours),
                         ("ngh_side", s.n_neighbours)):
                t[k] = t[k][:n]
            self._topo = t
        return self._topo

    def set_coeffs(self, conductivity=None, anisotropy=None, cross_section=None, sigma=None,
                   water_source_density=None, storativity=None):
        n = self.n_elements

        def arr(a, shape):
            if a is None:
                return None
            a = np.asarray(a, np.float64)
            if a.ndim == 0:
                a = np.full(shape, float(a))
            return np.ascontiguousarray(a.reshape(shape))

        keep = [arr(conductivity, n), arr(anisotropy, (n, 9)) if anisotropy is not None else None,
                arr(cross_section, n), arr(sigma, n), arr(water_source_density, n),
                arr(storativity, n)]
        c = _lib.Coeffs(*[ptr(a, C.c_double) for a in keep])
        check(lib.mh_set_coeffs(self.h, C.byref(c)), self.h)
        self._coeffs = keep

    def set_bc(self, bc_type, pressure=None, flux=None, robin_sigma=None):
        nb = self.n_boundaries
        keep = [i32(np.broadcast_to(np.asarray(bc_type, np.int32), (nb,)).copy())]
        for a in (pressure, flux, robin_sigma):
            keep.append(None if a is None else f64(np.broadcast_to(np.asarray(a, np.float64), (nb,)).copy()))
        b = _lib.BC(ptr(keep[0], C.c_int32), ptr(keep[1], C.c_double), ptr(keep[2], C.c_double),
                    ptr(keep[3], C.c_double))
        check(lib.mh_set_bc(self.h, C.byref(b)), self.h)
        self._bc = keep

    def assemble(self):
        check(lib.mh_assemble(self.h), self.h)

    def solve(self, **kw):
        o = solve_opts(**kw)
        st = _lib.SolveStats()
        rc = check(lib.mh_solve(self.h, C.byref(o), C.byref(st)), self.h)
        d = st.as_dict()
        d["status"] = rc
        return d

    def solution(self):
        out = np.zeros(self.sizes.mh_size)
        check(lib.mh_get_solution(self.h, ptr(out, C.c_double), len(out)), self.h)
        return out

    def element_flux(self):
        """Darcy flux vector at every element centre [n_elements, 3] from the last solution's
        side fluxes (DarcyFlowMHOutput::make_element_vector, darcy_flow_mh_output.cc:301-323)."""
        out = np.zeros((self.n_elements, 3))
        check(lib.mh_get_element_flux(self.h, ptr(out, C.c_double), out.size), self.h)
        return out

    def node_pressure(self):
        """Pressure at every node [n_nodes] from the last solution
        (DarcyFlowMHOutput::make_node_scalar_param, darcy_flow_mh_output.cc:424-546)."""
        out = np.zeros(self.sizes.n_nodes)
        check(lib.mh_get_node_pressure(self.h, ptr(out, C.c_double), len(out)), self.h)
        return out

    def water_balance(self, bdr_region, el_region, n_bdr_regions=None, n_el_regions=None):
        """Water balance of the last solution (DarcyFlowMHOutput::water_balance,
        darcy_flow_mh_output.cc:671-790) for region indices of the boundary objects (topology
        order) and of the elements: ([n_bdr_regions, 3] total, outflow, inflow;
        [n_el_regions] sources)."""
        br, er = i32(bdr_region), i32(el_region)
        nb = int(n_bdr_regions if n_bdr_regions is not None else (br.max() + 1 if br.size else 1))
        ne = int(n_el_regions if n_el_regions is not None else (er.max() + 1 if er.size else 1))
        bo, so = np.zeros((nb, 3)), np.zeros(ne)
        check(lib.mh_water_balance(self.h, ptr(br, C.c_int32), nb, ptr(er, C.c_int32), ne, ptr(bo, C.c_double),
                                   ptr(so, C.c_double)), self.h)
        return bo, so

    def transport_matrix(self, porosity=None):
        """Convection matrix of the explicit transport from the last solution's side fluxes
        (ConvectionTransport::create_transport_matrix_mpi, transport.cc:788-923): (row_ptr,
        col, val) CSR arrays [n_elements x n_elements] and cfl_max_step."""
        nnz = C.c_int64()
        check(lib.mh_transport_matrix(self.h, None, C.byref(nnz), None, None, None, None), self.h)
        rp = np.zeros(self.n_elements + 1, np.int32)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value)
        cfl = C.c_double()
        por = f64(porosity)
        check(lib.mh_transport_matrix(self.h, ptr(por, C.c_double), C.byref(nnz), ptr(rp, C.c_int32),
                                      ptr(col, C.c_int32), ptr(val, C.c_double), C.byref(cfl)), self.h)
        return (rp, col, val), cfl.value

    def schur_system(self):
        """The assembled edge system (reference schur2 after scale(-1)) as CSR + rhs."""
        s = self.sizes
        rp = np.zeros(s.n_edges + 1, np.int32)
        col = np.zeros(s.schur_nnz, np.int32)
        val = np.zeros(s.schur_nnz)
        rhs = np.zeros(s.n_edges)
        check(lib.mh_get_schur_system(self.h, ptr(rp, C.c_int32), ptr(col, C.c_int32),
                                      ptr(val, C.c_double), ptr(rhs, C.c_double)), self.h)
        return rp, col, val, rhs

    def unsteady_init(self, dt, init_pressure=None, lumped=False):
        ip = None if init_pressure is None else f64(np.broadcast_to(init_pressure, (self.n_elements,)).copy())
        check(lib.mh_unsteady_init(self.h, int(bool(lumped)), float(dt), ptr(ip, C.c_double)), self.h)

    def unsteady_step(self, dt, **kw):
        o = solve_opts(**kw)
        st = _lib.SolveStats()
        rc = check(lib.mh_unsteady_step(self.h, float(dt), C.byref(o), C.byref(st)), self.h)
        d = st.as_dict()
        d["status"] = rc
        return d

    # ---- aggregation multigrid (MH_SOLVER_AMG) ----
    def amg_info(self):
        """Levels of the last AMG solve: real rows and SELL slots per level."""
        cap = 32
        nl = np.zeros(1, np.int32)
        rows = np.zeros(cap, np.int64)
        slots = np.zeros(cap, np.int64)
        check(lib.mh_amg_info(self.h, ptr(nl, C.c_int32), rows.ctypes.data_as(C.POINTER(C.c_int64)),
                              slots.ctypes.data_as(C.POINTER(C.c_int64)), cap), self.h)
        n = int(nl[0])
        return dict(levels=n, rows=rows[:n].tolist(), slots=slots[:n].tolist())

    def amg_tail(self):
        """The coarse tail of the last AMG hierarchy's V-cycle: its first level and the CTAs of
        the cluster that runs it (0, 0: none)."""
        lv, cl = np.zeros(1, np.int32), np.zeros(1, np.int32)
        check(lib.mh_amg_tail(self.h, ptr(lv, C.c_int32), ptr(cl, C.c_int32)), self.h)
        return dict(level=int(lv[0]), cluster=int(cl[0]))

    def amg_level(self, level):
        """((row_ptr, col, val), agg, weight) of level `level` of the last AMG hierarchy."""
        n, nnz = C.c_int64(0), C.c_int64(0)
        check(lib.mh_amg_level(self.h, int(level), C.byref(n), C.byref(nnz), None, None, None, None, None), self.h)
        rp = np.zeros(n.value + 1, np.int32)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value, np.float32)
        agg = np.full(n.value, -1, np.int32)
        wt = np.ones(n.value, np.float32)
        check(lib.mh_amg_level(self.h, int(level), C.byref(n), C.byref(nnz), ptr(agg, C.c_int32), ptr(wt, C.c_float),
                               ptr(rp, C.c_int32), ptr(col, C.c_int32), ptr(val, C.c_float)), self.h)
        return (rp, col, val), agg, wt

    # ---- learned preconditioner (MH_SOLVER_FCG_LEARNED) ----
    def smoother_weights(self):
        """Per-edge weights of the multigrid's fine-level smoother (1 where none are set)."""
        w = np.zeros(self.n_edges, np.float32)
        check(lib.mh_smoother_weights_get(self.h, ptr(w, C.c_float), len(w)), self.h)
        return w

    def set_smoother_weights(self, w):
        """Fine-level smoother weights per edge (None: plain Jacobi-scaled smoothing)."""
        if w is None:
            check(lib.mh_smoother_weights_set(self.h, None, 0), self.h)
            return
        w = np.ascontiguousarray(w, np.float32)
        check(lib.mh_smoother_weights_set(self.h, ptr(w, C.c_float), len(w)), self.h)

    def learned_weights(self):
        w = np.zeros(_lib.MH_NN_PARAMS, np.float32)
        check(lib.mh_learned_get_weights(self.h, ptr(w, C.c_float), len(w)), self.h)
        return w

    def reset_learned(self):
        """The network's initial parameters (smoother weights 1) and a fresh optimiser state."""
        check(lib.mh_learned_reset(self.h), self.h)

    def set_learned_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        check(lib.mh_learned_set_weights(self.h, ptr(w, C.c_float), len(w)), self.h)

    def learned_grad(self, r, e):
        """Loss and parameter gradient of one pair (r, e) [n_edges], Jacobi-scaled space."""
        r, e = f64(r), f64(e)
        if len(r) != self.n_edges or len(e) != self.n_edges:
            raise ValueError("r and e need n_edges entries")
        g = np.zeros(_lib.MH_NN_PARAMS, np.float32)
        loss = C.c_double(0.0)
        check(lib.mh_learned_grad(self.h, ptr(r, C.c_double), ptr(e, C.c_double), ptr(g, C.c_float),
                                  C.byref(loss)), self.h)
        return loss.value, g

    def learned_grad_weights(self, r, e, refresh=True):
        """Loss, d loss / d smoother weight [n_edges] and the weights [n_edges] of one pair;
        refresh=False keeps the smoothing interval of the previous evaluation."""
        r, e = f64(r), f64(e)
        if len(r) != self.n_edges or len(e) != self.n_edges:
            raise ValueError("r and e need n_edges entries")
        dw = np.zeros(self.n_edges, np.float32)
        w = np.zeros(self.n_edges, np.float32)
        loss = C.c_double(0.0)
        check(lib.mh_learned_grad_weights(self.h, ptr(r, C.c_double), ptr(e, C.c_double), int(bool(refresh)),
                                          ptr(dw, C.c_float), ptr(w, C.c_float), C.byref(loss)), self.h)
        return loss.value, dw, w

    def learned_smoother(self):
        """The network's smoother weights [n_edges] for the assembled system."""
        w = np.zeros(self.n_edges, np.float32)
        check(lib.mh_learned_smoother(self.h, ptr(w, C.c_float), len(w)), self.h)
        return w

    def learned_apply(self, r):
        """z = M r [n_edges]: one V-cycle with the network's smoother weights."""
        r = f64(r)
        if len(r) != self.n_edges:
            raise ValueError("r needs n_edges entries")
        z = np.zeros(self.n_edges)
        check(lib.mh_learned_apply(self.h, ptr(r, C.c_double), ptr(z, C.c_double)), self.h)
        return z

    def learned_train(self, n_pairs=12, epochs=40, lr=2e-3, train_bias=False, solve_rtol=1e-9, seed=1):
        o = _lib.LearnOpts()
        lib.mh_learn_opts_default(C.byref(o))
        o.n_pairs, o.epochs, o.lr, o.train_bias = int(n_pairs), int(epochs), float(lr), int(bool(train_bias))
        o.solve_rtol, o.seed = float(solve_rtol), int(seed)
        st = _lib.LearnStats()
        check(lib.mh_learned_train(self.h, C.byref(o), C.byref(st)), self.h)
        return st.as_dict()

    # ---- MH_DofHandler accessors on a solution vector ----
    def split(self, sol):
        ns, ne = self.n_sides, self.n_elements
        return sol[:ns], sol[ns:ns + ne], sol[ns + ne:]


class MH_DofHandler:
    """Accessors of the MH solution layout [side fluxes | element pressures | edge pressures]."""

    def __init__(self, system, solution):
        self.sys = system
        self.sol = solution
        t = system.topology()
        self.el_side_start = t["el_side_start"]
        self.side_edge = t["side_edge"]

    def side_flux(self, element, local_side):
        return self.sol[self.el_side_start[element] + local_side]

    def side_scalar(self, element, local_side):
        e = self.side_edge[self.el_side_start[element] + local_side]
        return self.sol[self.sys.n_sides + self.sys.n_elements + e]

    def element_scalar(self, element):
        return self.sol[self.sys.n_sides + element]


def write_raw_output(path, solution, el_flux, el_side_start, side_edge, el_id=None, time=float("inf"),
                     append=False):
    """One "$FlowField" block of the flow field text output (DarcyFlowMHOutput::
    output_internal_flow_data, darcy_flow_mh_output.cc:793-829) from host arrays: the MH
    solution, the element flux vectors [n_el, 3], and the topology's el_side_start and
    side_edge; element ids default to the element indices.  The time defaults to inf, which is
    what the reference prints for a steady solve; unsteady output passes the step's time."""
    sol, ef = f64(solution), f64(el_flux)
    ss, se, ids = i32(el_side_start), i32(side_edge), i32(el_id)
    n_el = len(ss) - 1
    if ef.size != 3 * n_el:
        raise ValueError("el_flux needs 3 values per element")
    check(lib.mh_raw_output_write(str(path).encode(), int(bool(append)), float(time), n_el, ptr(ids, C.c_int32),
                                  ptr(ss, C.c_int32), ptr(se, C.c_int32), ptr(sol, C.c_double),
                                  ptr(ef, C.c_double)))


class DarcyFlowMH_Steady:
    """Steady MH Darcy flow with n_schurs = 2, solved on the GPU."""

    def __init__(self, mesh, coeffs, bc, solver=None):
        self.system = MHSystem(mesh)
        self.system.set_coeffs(**coeffs)
        self.system.set_bc(**bc)
        self.solver = dict(solver or {})
        self.stats = None
        self._solution = None

    def update_solution(self):
        self.system.assemble()
        self.stats = self.system.solve(**self.solver)
        self._solution = None
        return self.stats

    def get_solution_vector(self):
        if self._solution is None:
            self._solution = self.system.solution()
        return self._solution

    def get_mh_dofhandler(self):
        return MH_DofHandler(self.system, self.get_solution_vector())


class DarcyFlowMH_Unsteady(DarcyFlowMH_Steady):
    """Implicit Euler; time term -S|E|/dt on the element diagonal (darcy_flow_mh.cc:1614-1675)."""

    lumped = False

    def __init__(self, mesh, coeffs, bc, dt, init_pressure=None, solver=None):
        super().__init__(mesh, coeffs, bc, solver)
        self.dt = dt
        self.time = 0.0
        self.system.unsteady_init(dt, init_pressure, lumped=self.lumped)

    def update_solution(self, dt=None):
        dt = self.dt if dt is None else dt
        self.stats = self.system.unsteady_step(dt, **self.solver)
        self.time += dt
        self._solution = None
        return self.stats


class DarcyFlowLMH_Unsteady(DarcyFlowMH_Unsteady):
    """Lumped variant: time term on the edge rows (darcy_flow_mh.cc:1695-1827)."""

    lumped = True
