"""Meshes as flat arrays: the synthetic Kuhn cube meshes and gmsh 2.2 ASCII input (meshes and
$ElementData fields) through the library's parallel reader.

The gmsh reader follows GmshMeshReader (src/mesh/msh_gmshreader.cc:75-396): elements keep
file order; an element whose physical region name starts with '.' is a boundary element
(read_physical_names, msh_gmshreader.cc:220-244); element types 1/2/4/15 are lines,
triangles, tetrahedra and points.
"""
import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import lib, check


@dataclass
class Mesh:
    nodes: np.ndarray                      # (n_nodes, 3) float64
    el_dim: np.ndarray                     # (n_el,) int32
    el_nodes: np.ndarray                   # (n_el, 4) int32, -1 padded
    bc_dim: np.ndarray = None              # (n_bc,) int32
    bc_nodes: np.ndarray = None            # (n_bc, 4) int32
    el_region: np.ndarray = None           # physical region id per bulk element
    bc_region: np.ndarray = None           # physical region id per boundary element
    el_id: np.ndarray = None               # gmsh element ids
    region_names: dict = field(default_factory=dict)
    bc_id: np.ndarray = None               # gmsh ids of the boundary elements
    node_id: np.ndarray = None             # gmsh node ids
    el_partition: np.ndarray = None        # third element tag (0 if absent)
    regions: list = field(default_factory=list)  # (id, dim, boundary, name) in creation order

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, dtype=np.float64).reshape(-1, 3)
        self.el_dim = np.ascontiguousarray(self.el_dim, dtype=np.int32)
        self.el_nodes = np.ascontiguousarray(self.el_nodes, dtype=np.int32).reshape(-1, 4)
        if self.bc_dim is None:
            self.bc_dim = np.zeros(0, np.int32)
            self.bc_nodes = np.zeros((0, 4), np.int32)
        self.bc_dim = np.ascontiguousarray(self.bc_dim, dtype=np.int32)
        self.bc_nodes = np.ascontiguousarray(self.bc_nodes, dtype=np.int32).reshape(-1, 4)

    @property
    def n_elements(self):
        return len(self.el_dim)

    def desc(self):
        """mh_mesh_desc pointing into this mesh's arrays (keep the mesh alive while used)."""
        d = _lib.MeshDesc()
        d.n_nodes = len(self.nodes)
        d.node_xyz = _lib.ptr(self.nodes, C.c_double)
        d.n_elements = len(self.el_dim)
        d.el_dim = _lib.ptr(self.el_dim, C.c_int32)
        d.el_nodes = _lib.ptr(self.el_nodes, C.c_int32)
        d.n_bc_elements = len(self.bc_dim)
        d.bc_dim = _lib.ptr(self.bc_dim, C.c_int32) if len(self.bc_dim) else None
        d.bc_nodes = _lib.ptr(self.bc_nodes, C.c_int32) if len(self.bc_dim) else None
        return d

    def centres(self):
        """Element barycentres (Element::centre, src/mesh/elements.cc:139-150)."""
        n = self.el_dim + 1
        idx = np.where(self.el_nodes >= 0, self.el_nodes, 0)
        pts = self.nodes[idx]                                  # (n_el, 4, 3)
        mask = (np.arange(4)[None, :] < n[:, None])[..., None]
        return (pts * mask).sum(axis=1) / n[:, None]

    def bc_centres(self):
        if len(self.bc_dim) == 0:
            return np.zeros((0, 3))
        n = self.bc_dim + 1
        idx = np.where(self.bc_nodes >= 0, self.bc_nodes, 0)
        pts = self.nodes[idx]
        mask = (np.arange(4)[None, :] < n[:, None])[..., None]
        return (pts * mask).sum(axis=1) / n[:, None]


def concat_meshes(meshes):
    """Disjoint union of meshes (node indices shifted), in the order mh_create_batch uses."""
    nodes, dims, conn, bdims, bconn = [], [], [], [], []
    shift = 0
    for m in meshes:
        nodes.append(m.nodes)
        dims.append(m.el_dim)
        conn.append(np.where(m.el_nodes >= 0, m.el_nodes + shift, -1))
        bdims.append(m.bc_dim)
        bconn.append(np.where(m.bc_nodes >= 0, m.bc_nodes + shift, -1))
        shift += len(m.nodes)
    return Mesh(np.concatenate(nodes), np.concatenate(dims), np.concatenate(conn),
                np.concatenate(bdims), np.concatenate(bconn).reshape(-1, 4))


def cube_mesh(n, planes=(), lines=()):
    """Kuhn mesh of the unit cube (6 tetrahedra per cube of an n^3 grid).

    planes: iterable of (axis, grid_index) fracture planes (2n^2 triangles each).
    lines:  iterable of (axis, a, b) 1D channels along `axis` through grid indices (a, b) of the
            two other axes in increasing axis order (n segments each).
    """
    planes = list(planes)
    lines = list(lines)
    pa = np.array([p[0] for p in planes] or [0], np.int32)
    pi = np.array([p[1] for p in planes] or [0], np.int32)
    la = np.array([l[0] for l in lines] or [0], np.int32)
    l1 = np.array([l[1] for l in lines] or [0], np.int32)
    l2 = np.array([l[2] for l in lines] or [0], np.int32)
    h = C.c_void_p()
    check(lib.mh_cube_mesh_create(n, len(planes), _lib.ptr(pa, C.c_int32), _lib.ptr(pi, C.c_int32),
                                  len(lines), _lib.ptr(la, C.c_int32), _lib.ptr(l1, C.c_int32),
                                  _lib.ptr(l2, C.c_int32), C.byref(h)))
    try:
        d = _lib.MeshDesc()
        check(lib.mh_mesh_describe(h, C.byref(d)))
        nodes = np.ctypeslib.as_array(d.node_xyz, shape=(d.n_nodes * 3,)).reshape(-1, 3).copy()
        dim = np.ctypeslib.as_array(d.el_dim, shape=(d.n_elements,)).copy()
        eln = np.ctypeslib.as_array(d.el_nodes, shape=(d.n_elements * 4,)).reshape(-1, 4).copy()
    finally:
        lib.mh_mesh_destroy(h)
    return Mesh(nodes, dim, eln)


def _err_buf():
    return C.create_string_buffer(1024)


def _raise(rc, err):
    msg = err.value.decode(errors="replace")
    if rc == _lib.MH_ERR_IO:
        raise OSError(msg)
    if rc == _lib.MH_ERR_NOMEM:
        raise MemoryError(msg)
    raise ValueError(msg)


def read_gmsh(path):
    """Reads a gmsh 2.2 ASCII mesh with the library's parallel reader (mh_gmsh_read; the rules
    of GmshMeshReader::read_mesh, src/mesh/msh_gmshreader.cc:75-244, and RegionDB::add_region,
    src/mesh/region.cc:107-175).  Bulk and boundary elements keep file order; node indices
    refer to the file's node order.  Raises OSError when the file cannot be read and
    ValueError (with the file line) for a format error."""
    h = C.c_void_p()
    err = _err_buf()
    rc = lib.mh_gmsh_read(os.fsencode(str(path)), C.byref(h), err, len(err))
    if rc != _lib.MH_OK:
        _raise(rc, err)
    try:
        d = _lib.MeshDesc()
        check(lib.mh_mesh_describe(h, C.byref(d)))
        g = _lib.GmshInfo()
        check(lib.mh_gmsh_info_get(h, C.byref(g)))
        arr = lambda p, n, shape=None: (np.ctypeslib.as_array(p, shape=(n,)).copy() if n else
                                        np.zeros(0, np.dtype(p._type_)))
        nn, ne, nb = d.n_nodes, d.n_elements, d.n_bc_elements
        m = Mesh(arr(d.node_xyz, nn * 3).reshape(-1, 3), arr(d.el_dim, ne), arr(d.el_nodes, ne * 4).reshape(-1, 4),
                 arr(d.bc_dim, nb) if nb else None, arr(d.bc_nodes, nb * 4).reshape(-1, 4) if nb else None)
        m.el_region = arr(g.el_region, ne)
        m.el_id = arr(g.el_id, ne)
        m.el_partition = arr(g.el_partition, ne)
        m.bc_region = arr(g.bc_region, nb)
        m.bc_id = arr(g.bc_id, nb)
        m.node_id = arr(g.node_id, nn)
        m.regions = [(g.region_id[i], g.region_dim[i], bool(g.region_boundary[i]), g.region_name[i].decode())
                     for i in range(g.n_regions)]
        m.region_names = {r[0]: r[3] for r in m.regions}
    finally:
        lib.mh_mesh_destroy(h)
    return m


def read_element_data(path, field_name, el_ids, time=0.0, n_components=1):
    """Values of the element field `field_name` of a gmsh 2.2 file at `time`, for the elements
    with ids `el_ids` (strictly ascending, e.g. Mesh.el_id): an array [len(el_ids),
    n_components] in that order, ready for MHSystem.set_coeffs.  The library's reader
    (mh_gmsh_element_data) follows GmshMeshReader::read_element_data
    (src/mesh/msh_gmshreader.cc:306-396): the $ElementData sections of the field are taken in
    file order, each one whose time is <= time (1 + 2 eps) overwriting the elements it lists;
    a data line is "id v_1 .. v_n", ids that are not among el_ids are skipped, and an element
    no section lists is NaN.  Raises ValueError when the file has no section of the field,
    when none is at or before `time`, or when a row that is read has fewer than n_components
    values; OSError when the file cannot be read."""
    ids = np.ascontiguousarray(el_ids, dtype=np.int64)
    out = np.empty((ids.size, n_components), np.float64)
    err = _err_buf()
    rc = lib.mh_gmsh_element_data(os.fsencode(str(path)), field_name.encode(), float(time), ids.size,
                                  ids.ctypes.data, int(n_components), out.ctypes.data, err, len(err))
    if rc != _lib.MH_OK:
        _raise(rc, err)
    return out
