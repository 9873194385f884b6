"""The product's C++ topology builder (edges, boundaries, VB neighbours) is identical to the
pure-Python restatement of Mesh::make_neighbours_and_edges (no GPU)."""
import ctypes as C

import numpy as np
import pytest

import mhdarcy
import topology as T
from helpers import load_fixture
from mhdarcy import _lib

KEYS = ("el_side_start", "side_edge", "side_bdr", "bdr_bc_element", "bdr_edge", "ngh_element", "ngh_edge",
        "ngh_side")


def compare(mesh):
    ref = T.build(mesh)
    with mhdarcy.MHSystem(mesh) as s:
        t = s.topology()
        assert s.n_edges == ref["n_edges"]
        for k in KEYS:
            assert np.array_equal(t[k], ref[k]), k
        return s.sizes


@pytest.mark.parametrize("name", ["t01", "t02", "t03", "t05_robin", "t06_32", "t06_21", "t08", "t10_mh", "t13", "t14"])
def test_fixture_topology(name):
    z, mesh = load_fixture(name)
    compare(mesh)


@pytest.mark.parametrize("n,planes,lines", [
    (3, [(2, 1)], [(0, 1, 1)]),
    (4, [(0, 2), (2, 2)], [(1, 2, 2)]),                 # channel on the intersection of two planes
    (4, [(0, 1), (1, 3), (2, 2)], [(2, 1, 3), (0, 3, 2)]),
    (2, [], []),
])
def test_cube_topology(n, planes, lines):
    mesh = mhdarcy.cube_mesh(n, planes, lines)
    compare(mesh)


@pytest.mark.parametrize("n", [8, 16])
def test_cube_sizes_match_formulas(n):
    """Tets 6n^3, faces 12n^3+6n^2; a z-plane fracture adds 2n^2 triangles, 2n^2 split faces and
    3n^2+2n segment edges; an x-line adds n segments, n+1 point edges and n split edges."""
    mesh = mhdarcy.cube_mesh(n, [(2, n // 2)], [(0, n // 2, n // 2)])
    with mhdarcy.MHSystem(mesh) as s:
        z = s.sizes
        assert z.n_el_dim[3] == 6 * n ** 3 and z.n_el_dim[2] == 2 * n * n and z.n_el_dim[1] == n
        assert z.n_sides == 4 * 6 * n ** 3 + 3 * 2 * n * n + 2 * n
        assert z.n_edges == 12 * n ** 3 + 6 * n * n + 2 * n * n + 3 * n * n + 2 * n + (n + 1) + n
        assert z.n_neighbours == 2 * 2 * n * n + 2 * n
        assert z.mh_size == z.n_sides + z.n_elements + z.n_edges
        # every edge row couples with itself and the other sides of its elements
        assert 6 * z.n_edges < z.schur_nnz < 8 * z.n_edges


def test_boundary_element_matching_bulk_element_is_rejected():
    z, mesh = load_fixture("t06_32")
    # declare a bulk triangle as a boundary element as well
    tri = np.nonzero(mesh.el_dim == 2)[0][0]
    bad = mhdarcy.Mesh(mesh.nodes, mesh.el_dim, mesh.el_nodes, np.array([2], np.int32),
                       mesh.el_nodes[tri:tri + 1].copy())
    with pytest.raises(mhdarcy.MHError) as ei:
        mhdarcy.MHSystem(bad)
    assert ei.value.status == _lib.MH_ERR_TOPOLOGY


def test_invalid_node_index_is_rejected():
    mesh = mhdarcy.cube_mesh(1)
    mesh.el_nodes[0, 0] = 10_000
    with pytest.raises(mhdarcy.MHError) as ei:
        mhdarcy.MHSystem(mesh)
    assert ei.value.status == _lib.MH_ERR_INVALID


def test_gmsh_reader_round_trip(tmp_path):
    """A fixture mesh written as gmsh 2.2 and read back by the library's reader: one physical
    region per dimension (a region has one dimension), boundary regions named with '.'."""
    z, mesh = load_fixture("t06_21")
    path = tmp_path / "m.msh"
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", "4", '2 1 "plane"', '1 2 "channel"',
             '1 3 ".bnd_lines"', '0 4 ".bnd_points"', "$EndPhysicalNames", "$Nodes", str(len(mesh.nodes))]
    lines += ["%d %.17g %.17g %.17g" % (i + 1, *p) for i, p in enumerate(mesh.nodes)]
    lines += ["$EndNodes", "$Elements", str(len(mesh.el_dim) + len(mesh.bc_dim))]
    typ = {0: 15, 1: 1, 2: 2, 3: 4}
    bulk_region, bc_region = {2: 1, 1: 2}, {1: 3, 0: 4}
    k = 1
    for d, nd in zip(mesh.bc_dim, mesh.bc_nodes):
        r = bc_region[d]
        lines.append("%d %d 2 %d %d %s" % (k, typ[d], r, r, " ".join(str(v + 1) for v in nd[:d + 1])))
        k += 1
    for d, nd in zip(mesh.el_dim, mesh.el_nodes):
        r = bulk_region[d]
        lines.append("%d %d 2 %d %d %s" % (k, typ[d], r, r, " ".join(str(v + 1) for v in nd[:d + 1])))
        k += 1
    lines.append("$EndElements")
    path.write_text("\n".join(lines) + "\n")
    m2 = mhdarcy.read_gmsh(str(path))
    assert np.array_equal(m2.el_nodes, mesh.el_nodes) and np.array_equal(m2.bc_nodes, mesh.bc_nodes)
    assert np.allclose(m2.nodes, mesh.nodes, rtol=0, atol=0)


@pytest.mark.parametrize("name", ["t01", "t02", "t03", "t05_robin", "t06_32", "t06_21", "t08", "t10_mh", "t13", "t14"])
def test_oracle_c_topology_matches_python_restatement(name):
    """The oracle's C topology (used by the CPU arm of the benchmark, which loads no product
    code) equals the pure-Python restatement on every fixture, explicit boundary elements
    included."""
    import cases as OC
    z, mesh = load_fixture(name)
    ref = T.build(mesh)
    t = OC.topology(mesh)
    assert t["n_edges"] == ref["n_edges"]
    for k in KEYS:
        assert np.array_equal(t[k], ref[k]), k


@pytest.mark.parametrize("cfg,n,seed", [(1, 6, None), (2, 8, None), (3, None, 77), (4, 6, None), (5, 16, None)])
def test_oracle_cases_match_library_cases(cfg, n, seed):
    """The CPU arm's numpy Kuhn cube and C topology give the library's mesh, coefficients and
    topology element for element (the two benchmark arms solve identical inputs)."""
    import cases as OC
    from mhdarcy.cases import make_case
    m1, c1 = make_case(cfg, seed=seed, n=n)
    m2, c2 = OC.make_case(cfg, seed=seed, n=n)
    assert np.array_equal(m1.nodes, m2.nodes)
    assert np.array_equal(m1.el_dim, m2.el_dim) and np.array_equal(m1.el_nodes, m2.el_nodes)
    assert sorted(c1) == sorted(c2)
    for k in c1:
        assert np.array_equal(c1[k], c2[k]), k
    t2 = OC.topology(m2)
    with mhdarcy.MHSystem(m1) as s:
        t1 = s.topology()
        assert s.n_edges == t2["n_edges"]
    for k in KEYS:
        assert np.array_equal(t1[k], t2[k]), k


def test_oracle_c_topology_rejects_boundary_on_bulk_element():
    import cases as OC
    z, mesh = load_fixture("t06_32")
    tri = np.nonzero(mesh.el_dim == 2)[0][0]
    bad = mhdarcy.Mesh(mesh.nodes, mesh.el_dim, mesh.el_nodes, np.array([2], np.int32),
                       mesh.el_nodes[tri:tri + 1].copy())
    with pytest.raises(ValueError):
        OC.topology(bad)
