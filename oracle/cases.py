"""TEST INFRASTRUCTURE ONLY: the benchmark problems built without the GPU library, for
bench.py's CPU arm and the tests.

* cube_mesh  -- the Kuhn cube mesh (6 tetrahedra per grid cube, one per permutation of the
                axes, from the low corner to the high corner), fracture planes made of the
                coincident tetrahedron faces and 1D channels along grid lines, in numpy.  It
                must equal the library's mesh element for element (tests/test_topology.py).
* topology   -- the C restatement of Mesh::make_neighbours_and_edges (orc_mesh.c).
* make_case  -- the seeded coefficients of the benchmark configurations, taken from the
                package's own case module (loaded by file path, without the package's native
                library) with this module's mesh builder, so both sides solve the same inputs.
* problem    -- make_case + topology + the Dirichlet x boundary data as an oracle.Problem.
It is never imported by the product.
"""
import ctypes as C
import importlib.util
import os

import numpy as np

import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
_CASES_PY = os.path.join(_HERE, "..", "svn-export_b200", "mhdarcy", "cases.py")


class CubeMesh:
    """Flat mesh arrays with the attributes the case generator and oracle.Problem read."""

    def __init__(self, nodes, el_dim, el_nodes):
        self.nodes = np.ascontiguousarray(nodes, np.float64)
        self.el_dim = np.ascontiguousarray(el_dim, np.int32)
        self.el_nodes = np.ascontiguousarray(el_nodes, np.int32)
        self.bc_dim = np.zeros(0, np.int32)
        self.bc_nodes = np.zeros((0, 4), np.int32)

    @property
    def n_elements(self):
        return len(self.el_dim)

    def centres(self):
        n = self.el_dim + 1
        idx = np.where(self.el_nodes >= 0, self.el_nodes, 0)
        pts = self.nodes[idx]
        mask = (np.arange(4)[None, :] < n[:, None])[..., None]
        return (pts * mask).sum(axis=1) / n[:, None]


def cube_mesh(n, planes=(), lines=()):
    """Kuhn mesh of the unit cube with n^3 grid cubes.  Node (i, j, k) has index
    i + (n+1)(j + (n+1)k) and coordinates (i, j, k)/n.  Elements: the 6 tetrahedra of every
    cube (cubes x-fastest; tetrahedron t walks from the low corner along the axes of the t-th
    permutation (012, 021, 102, 120, 201, 210) to the high corner); then per fracture plane
    (axis, index) its 2n^2 triangles (squares fastest along the lower remaining axis u, each
    split by the diagonal from its low to its high corner: (00, 10, 11) and (00, 01, 11) in
    (u, w)); then per channel (axis, a, b) its n segments."""
    n1 = n + 1
    ii, jj, kk = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    nodes = np.empty((n1 ** 3, 3))
    idx = (ii + n1 * (jj + n1 * kk)).ravel()
    nodes[idx, 0] = ii.ravel() / n
    nodes[idx, 1] = jj.ravel() / n
    nodes[idx, 2] = kk.ravel() / n
    node = lambda c: c[..., 0] + n1 * (c[..., 1] + n1 * c[..., 2])
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)           # cubes, x fastest
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = np.empty((len(base), 6, 4), np.int64)
    for t, p in enumerate(perms):
        c = base.copy()
        tets[:, t, 0] = node(c)
        c[:, p[0]] += 1
        tets[:, t, 1] = node(c)
        c[:, p[1]] += 1
        tets[:, t, 2] = node(c)
        tets[:, t, 3] = node(base + 1)
    parts_nodes = [tets.reshape(-1, 4)]
    parts_dim = [np.full(6 * n ** 3, 3)]
    for ax, pos in planes:
        u, w = sorted(((ax + 1) % 3, (ax + 2) % 3))
        b, a = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        a, b = a.ravel(), b.ravel()

        def corner(du, dw):
            c = np.zeros((len(a), 3), np.int64)
            c[:, ax] = pos
            c[:, u] = a + du
            c[:, w] = b + dw
            return node(c)
        c00, c10, c11, c01 = corner(0, 0), corner(1, 0), corner(1, 1), corner(0, 1)
        tri = np.full((len(a), 2, 4), -1, np.int64)
        tri[:, 0, :3] = np.stack([c00, c10, c11], axis=1)
        tri[:, 1, :3] = np.stack([c00, c01, c11], axis=1)
        parts_nodes.append(tri.reshape(-1, 4))
        parts_dim.append(np.full(2 * n * n, 2))
    for ax, la, lb in lines:
        u, w = sorted(((ax + 1) % 3, (ax + 2) % 3))
        s = np.arange(n)
        c0 = np.zeros((n, 3), np.int64)
        c0[:, ax] = s
        c0[:, u] = la
        c0[:, w] = lb
        c1 = c0.copy()
        c1[:, ax] += 1
        seg = np.full((n, 4), -1, np.int64)
        seg[:, 0] = node(c0)
        seg[:, 1] = node(c1)
        parts_nodes.append(seg)
        parts_dim.append(np.full(n, 1))
    return CubeMesh(nodes, np.concatenate(parts_dim), np.concatenate(parts_nodes))


def topology(mesh):
    """Topology of a mesh by the C restatement (orc_topology): the arrays of the library's
    mh_get_topology plus n_edges."""
    L = O.lib
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    dim, eln = i32(mesh.el_dim), i32(mesh.el_nodes).reshape(-1)
    bcd, bcn = i32(mesh.bc_dim), i32(mesh.bc_nodes).reshape(-1)
    ne, nb = len(dim), len(bcd)
    ns = int(np.sum(dim.astype(np.int64) + 1))
    out = {k: np.zeros(sz, np.int32) for k, sz in (("el_side_start", ne + 1), ("side_edge", ns),
                                                    ("side_bdr", ns), ("bdr_bc_element", ns + nb),
                                                    ("bdr_edge", ns + nb), ("ngh_element", ns),
                                                    ("ngh_edge", ns), ("ngh_side", ns))}
    counts = np.zeros(3, np.int64)
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    rc = L.orc_topology(len(mesh.nodes), ne, p(dim), p(eln), nb, p(bcd) if nb else None, p(bcn) if nb else None,
                        p(out["el_side_start"]), p(out["side_edge"]), p(out["side_bdr"]), p(out["bdr_bc_element"]),
                        p(out["bdr_edge"]), p(out["ngh_element"]), p(out["ngh_edge"]), p(out["ngh_side"]),
                        counts.ctypes.data_as(C.POINTER(C.c_int64)))
    if rc:
        raise ValueError("orc_topology failed (%d)" % rc)
    ned, nbd, nng = (int(c) for c in counts)
    for k in ("bdr_bc_element", "bdr_edge"):
        out[k] = out[k][:nbd].copy()
    for k in ("ngh_element", "ngh_edge", "ngh_side"):
        out[k] = out[k][:nng].copy()
    out["n_edges"] = ned
    return out


def _cases_module():
    spec = importlib.util.spec_from_file_location("mh_bench_cases", _CASES_PY)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_case(cfg, seed=None, n=None):
    """Mesh and coefficients of benchmark configuration cfg, identical to the package's
    mhdarcy.cases.make_case (same seeds), with this module's mesh builder."""
    return _cases_module().make_case(cfg, seed=seed, n=n, mesh_builder=cube_mesh)


def problem(cfg, seed=None, n=None):
    """(Problem, mesh, coeffs, topology, bc) of configuration cfg: Dirichlet p=1 at x=0 and p=0
    at x=1, homogeneous Neumann elsewhere (the benchmark's boundary data)."""
    mod = _cases_module()
    mesh, coeffs = mod.make_case(cfg, seed=seed, n=n, mesh_builder=cube_mesh)
    topo = topology(mesh)
    bc, _ = mod.dirichlet_x_bc(topo, mesh)
    P = O.Problem(mesh, topo, topo["n_edges"], conductivity=coeffs["conductivity"],
                  cross_section=coeffs["cross_section"], storativity=coeffs.get("storativity", 1.0),
                  bc_type=bc["bc_type"], bc_pressure=bc["pressure"])
    return P, mesh, coeffs, topo, bc
