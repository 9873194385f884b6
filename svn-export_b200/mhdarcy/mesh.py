"""Meshes as flat arrays: the synthetic Kuhn cube meshes and a gmsh 2.2 ASCII reader.

The gmsh reader follows GmshMeshReader (src/mesh/msh_gmshreader.cc:125-260): elements keep
file order; an element whose physical region name starts with '.' is a boundary element
(read_physical_names, msh_gmshreader.cc:242-262); element types 1/2/4/15 are lines,
triangles, tetrahedra and points.
"""
import ctypes as C
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


def read_gmsh(path):
    """Reads a gmsh 2.2 ASCII mesh (nodes, elements, physical names)."""
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    names = {}
    node_ids = []
    coords = []
    bulk = []
    bnd = []
    boundary_regions = set()
    while i < len(lines):
        s = lines[i].strip()
        if s == "$PhysicalNames":
            n = int(lines[i + 1])
            for k in range(n):
                parts = lines[i + 2 + k].split(None, 2)
                dim, rid, name = int(parts[0]), int(parts[1]), parts[2].strip().strip('"')
                names[rid] = name
                if name.startswith("."):
                    boundary_regions.add(rid)
            i += n + 2
        elif s == "$Nodes":
            n = int(lines[i + 1])
            for k in range(n):
                p = lines[i + 2 + k].split()
                node_ids.append(int(p[0]))
                coords.append([float(p[1]), float(p[2]), float(p[3])])
            i += n + 2
        elif s == "$Elements":
            n = int(lines[i + 1])
            nmap = {nid: k for k, nid in enumerate(node_ids)}
            tdim = {1: 1, 2: 2, 4: 3, 15: 0}
            for k in range(n):
                p = [int(v) for v in lines[i + 2 + k].split()]
                eid, etype, ntags = p[0], p[1], p[2]
                dim = tdim[etype]
                region = p[3]
                nd = [nmap[v] for v in p[3 + ntags:3 + ntags + dim + 1]]
                nd = nd + [-1] * (4 - len(nd))
                rec = (eid, dim, nd, region)
                if region in boundary_regions:
                    bnd.append(rec)
                elif dim > 0:
                    bulk.append(rec)
            i += n + 2
        else:
            i += 1
    m = Mesh(np.array(coords), np.array([r[1] for r in bulk], np.int32),
             np.array([r[2] for r in bulk], np.int32),
             np.array([r[1] for r in bnd], np.int32) if bnd else None,
             np.array([r[2] for r in bnd], np.int32).reshape(-1, 4) if bnd else None)
    m.el_region = np.array([r[3] for r in bulk], np.int32)
    m.bc_region = np.array([r[3] for r in bnd], np.int32)
    m.el_id = np.array([r[0] for r in bulk], np.int64)
    m.region_names = names
    return m


def _data_header(lines, i):
    """Parses the tags of an $ElementData header starting at line i (the string-tag count):
    field name, time, component and entity counts, and the index of the first data line
    (GmshMeshReader::read_data_header, src/mesh/msh_gmshreader.cc:251-303).  Missing tags
    take the reference's defaults: time 0, one component, zero entities."""
    n_str = int(lines[i].split()[0])
    name = lines[i + 1].strip().strip('"') if n_str > 0 else ""
    i += 1 + n_str
    n_real = int(lines[i].split()[0])
    time = float(lines[i + 1].split()[0]) if n_real > 0 else 0.0
    i += 1 + n_real
    n_int = int(lines[i].split()[0])
    ints = [int(lines[i + 1 + k].split()[0]) for k in range(n_int)]
    i += 1 + n_int
    n_comp = ints[1] if n_int > 1 else 1
    n_ent = ints[2] if n_int > 2 else 0
    return name, time, n_comp, n_ent, i


def read_element_data(path, field_name, el_ids, time=0.0, n_components=1):
    """Values of the element field `field_name` of a gmsh 2.2 file at `time`, for the elements
    with ids `el_ids` (ascending, e.g. Mesh.el_id): an array [len(el_ids), n_components] in that
    order, ready for MHSystem.set_coeffs.  Follows GmshMeshReader::read_element_data
    (src/mesh/msh_gmshreader.cc:306-396): the $ElementData sections of the field are taken in
    file order, and the last one whose time is <= time (1 + 2 eps) gives the values; a data line
    is "id v_1 .. v_n" with ids ascending, ids that are not among el_ids are skipped, and an
    element without a line keeps the value of an earlier section (NaN if none had it).  A
    section with another component count is read with n_components values per line, as the
    reference does.  Raises ValueError when the file has no section of the field, when none is at
    or before `time` (the reference then leaves the field's values unset), or when a row has
    fewer values than n_components."""
    ids = np.asarray(el_ids, np.int64)
    if ids.size > 1 and np.any(np.diff(ids) <= 0):
        raise ValueError("el_ids must be ascending")
    with open(path) as f:
        lines = f.read().split("\n")
    out = np.full((ids.size, n_components), np.nan)
    found = used = False
    limit = time * (1.0 + 2.0 * np.finfo(float).eps)
    i = 0
    while i < len(lines):
        if lines[i].strip() != "$ElementData":
            i += 1
            continue
        name, t, _, n_ent, i = _data_header(lines, i + 1)
        if name != field_name:
            continue
        found = True
        if t > limit:
            break
        used = True
        pos = 0
        for row in lines[i:i + n_ent]:
            p = row.split()
            eid = int(p[0])
            while pos < ids.size and ids[pos] < eid:
                pos += 1
            if pos == ids.size:
                break  # an id past the last element: the rest of the section is skipped
            if ids[pos] == eid:
                if len(p) - 1 < n_components:
                    raise ValueError(f"{path}: element {eid} of field '{field_name}' has {len(p) - 1} values, "
                                     f"{n_components} expected")
                out[pos] = [float(v) for v in p[1:1 + n_components]]
        i += n_ent
    if not found:
        raise ValueError(f"{path}: no $ElementData section for field '{field_name}'")
    if not used:
        raise ValueError(f"{path}: no $ElementData of field '{field_name}' at or before time {time}")
    return out
