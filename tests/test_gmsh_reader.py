"""The library's parallel gmsh 2.2 reader (mh_gmsh_read, mh_gmsh_element_data) against the
sequential restatement of the reference's GmshMeshReader, RegionDB and Tokenizer
(oracle/gmsh.py), on files written here: the golden fixtures' meshes, sparse and shuffled ids,
comments, blank lines, CRLF, quoted names, partitions and extra tags, unnamed regions, points
in bulk regions, and files large enough for the multi-threaded line index.  The arrays agree
bit for bit, and every error the reference raises is raised for the same first offending line
of the file (no GPU)."""
import re

import numpy as np
import pytest

import gmsh as G
import mhdarcy
from helpers import load_fixture

TYPE = {0: 15, 1: 1, 2: 2, 3: 4}
KEYS = ("nodes", "node_id", "el_id", "el_dim", "el_nodes", "el_region", "el_partition", "bc_id", "bc_dim",
        "bc_nodes", "bc_region")


def mesh_lines(nodes, node_ids, elements, names, nl="\n", sep=" ", comments=False):
    """gmsh 2.2 text; elements are (id, type, tags, node ids), names (dim, id, name)."""
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat"]
    if names:
        out += ["$PhysicalNames", str(len(names))]
        out += ['%d%s%d%s"%s"' % (d, sep, i, sep, n) for d, i, n in names]
        out += ["$EndPhysicalNames"]
    out += ["$Nodes", str(len(nodes))]
    for k, (i, p) in enumerate(zip(node_ids, nodes)):
        out.append(sep.join(["%d" % i] + ["%.17g" % v for v in p]))
        if comments and k % 7 == 3:
            out += ["# a comment line", "", "   "]
    out += ["$EndNodes", "$Elements", str(len(elements))]
    for k, (i, t, tags, nd) in enumerate(elements):
        out.append(sep.join(str(v) for v in [i, t, len(tags), *tags, *nd]))
        if comments and k % 5 == 1:
            out += ["\t# indented comment", ""]
    out += ["$EndElements"]
    return nl.join(out) + nl


def fixture_file(name):
    """(nodes, elements, names) of a golden fixture's mesh, one physical region per region id."""
    z, mesh = load_fixture(name)
    elements, names, seen = [], [], {}
    k = 1
    for dims, nds, regs, bnd in ((z["bc_dim"], z["bc_nodes"], z["bc_region"], True),
                                 (z["el_dim"], z["el_nodes"], z["el_region"], False)):
        for d, nd, r in zip(dims, nds, regs):
            if int(r) not in seen:
                seen[int(r)] = d
                names.append((int(d), int(r), (".b%d" if bnd else "r%d") % r))
            elements.append((k, TYPE[int(d)], [int(r), int(r)], [int(v) + 1 for v in nd[:d + 1]]))
            k += 1
    return mesh, z["nodes"], elements, names


def compare(path):
    ref = G.read_mesh(str(path))
    got = mhdarcy.read_gmsh(str(path))
    for k in KEYS:
        a = getattr(got, k)
        a = np.zeros(0) if a is None else a
        assert a.dtype == ref[k].dtype or a.size == 0, k
        assert np.array_equal(a, ref[k]), k
    assert got.regions == ref["regions"]
    return got, ref


@pytest.mark.parametrize("name", ["t01", "t02", "t03", "t05_robin", "t06_32", "t08", "t13"])
def test_fixture_meshes(tmp_path, name):
    mesh, nodes, elements, names = fixture_file(name)
    p = tmp_path / "m.msh"
    p.write_text(mesh_lines(nodes, range(1, len(nodes) + 1), elements, names))
    got, _ = compare(p)
    assert np.array_equal(got.nodes, mesh.nodes) and np.array_equal(got.el_nodes, mesh.el_nodes)
    assert np.array_equal(got.el_dim, mesh.el_dim)
    if mesh.bc_dim is not None and len(mesh.bc_dim):
        assert np.array_equal(got.bc_dim, mesh.bc_dim) and np.array_equal(got.bc_nodes, mesh.bc_nodes)


def test_format_variants(tmp_path):
    """Sparse shuffled node ids, CRLF, tabs and runs of blanks, comment and blank lines, quoted
    names with blanks, four tags (partition), an unnamed region, points in a bulk region."""
    mesh, nodes, elements, names = fixture_file("t03")
    rng = np.random.default_rng(0)
    ids = rng.permutation(np.arange(1, 40 * len(nodes), 40))[:len(nodes)]
    elements = [(i, t, tags + [5 + i % 3, 9], [int(ids[v - 1]) for v in nd]) for i, t, tags, nd in elements]
    names = [(d, r, n.replace("r", "bulk region ")) for d, r, n in names]
    # an unnamed 2D region and points in a bulk (unnamed) region
    elements[-1] = (elements[-1][0], elements[-1][1], [77, 1, 3], elements[-1][3])
    elements.append((90001, 15, [78, 1], [int(ids[0])]))
    elements.append((90002, 15, [78, 1], [int(ids[1])]))
    for nl, sep in (("\r\n", "\t"), ("\n", "  \t "), ("\n", " ")):
        p = tmp_path / "v.msh"
        p.write_bytes(mesh_lines(nodes, ids, elements, names, nl=nl, sep=sep, comments=True).encode())
        got, ref = compare(p)
    assert (77, 2, False, "region_77") in got.regions and (78, 0, False, "region_78") in got.regions
    assert 90001 not in got.el_id and 90001 not in got.bc_id      # points in bulk regions are dropped
    assert got.el_region[-1] == 77 and got.el_partition[-1] == 3
    assert set(got.el_partition[:-1]) == {5, 6, 7}
    assert any(" " in n for _, _, _, n in got.regions)
    assert np.array_equal(got.node_id, ids)
    assert np.array_equal(got.nodes, mesh.nodes)


def test_large_file_uses_threads(tmp_path):
    """A file above 1 MiB (the line index and every row loop run multi-threaded) with
    shuffled, sparse node ids: identical to the sequential restatement."""
    cube = mhdarcy.cube_mesh(18, [(2, 9)], [(0, 9, 9)])
    rng = np.random.default_rng(1)
    ids = rng.permutation(len(cube.nodes)) * 3 + 11
    elements = []
    for k, (d, nd) in enumerate(zip(cube.el_dim, cube.el_nodes)):
        elements.append((k + 1, TYPE[int(d)], [int(d), 100 + k % 4], [int(ids[v]) for v in nd[:d + 1]]))
    names = [(3, 3, "rock"), (2, 2, "fracture"), (1, 1, "channel")]
    p = tmp_path / "big.msh"
    p.write_text(mesh_lines(cube.nodes, ids, elements, names))
    assert p.stat().st_size > (1 << 20)
    got, _ = compare(p)
    assert np.array_equal(got.el_nodes, cube.el_nodes) and np.array_equal(got.nodes, cube.nodes)


BASE = """$MeshFormat
2.2 0 8
$EndMeshFormat
$PhysicalNames
3
2 1 "plane"
1 2 ".edge"
2 3 "other"
$EndPhysicalNames
$Nodes
4
1 0 0 0
2 1 0 0
3 1 1 0
4 0 1 0
$EndNodes
$Elements
4
1 2 2 1 1 1 2 3
2 2 2 1 1 1 3 4
3 1 2 2 2 1 2
4 2 2 3 3 2 3 4
$EndElements
"""


def edit(text, old, new):
    assert old in text
    return text.replace(old, new, 1)


ERRORS = [
    ("unsupported type", lambda t: edit(t, "2 2 2 1 1 1 3 4", "2 3 2 1 1 1 3 4")),
    ("fewer than two tags", lambda t: edit(t, "2 2 2 1 1 1 3 4", "2 2 1 1 1 3 4")),
    ("unknown node id 9", lambda t: edit(t, "2 2 2 1 1 1 3 4", "2 2 2 1 1 1 3 9")),
    ("repeated node id", lambda t: edit(t, "3 1 1 0\n", "2 1 1 0\n")),
    ("repeated element id", lambda t: edit(t, "2 2 2 1 1 1 3 4", "1 2 2 1 1 1 3 4")),
    ("element of dimension 1", lambda t: edit(t, "3 1 2 2 2 1 2", "3 1 2 1 2 1 2")),
    ("already names", lambda t: edit(t, '2 3 "other"', '2 1 "other"')),
    ("already belongs", lambda t: edit(t, '2 3 "other"', '2 3 "plane"')),
    ("given dimensions", lambda t: edit(t, '2 3 "other"', '1 1 "plane"\n2 3 "other"').replace("3\n2 1", "4\n2 1", 1)),
    ("wrong format", lambda t: edit(t, "2 1 0 0\n", "2 1.0.0 0 0\n")),
    ("wrong format", lambda t: edit(t, "2 1 0 0\n", "2 1 0\n")),
    ("wrong format", lambda t: edit(t, "4 2 2 3 3 2 3 4", "4 2 2 3 3 2 3")),
    ("wrong format", lambda t: edit(t, "2 1 0 0\n", "2 1e999 0 0\n")),
    ("zero number of nodes", lambda t: edit(t, "$Nodes\n4\n", "$Nodes\n0\n")),
    # counts beyond the rows of the file: the first line that is not a row is the error
    ("wrong format", lambda t: edit(t, "$Nodes\n4\n", "$Nodes\n2000000000\n")),
    ("wrong format", lambda t: edit(t, "$Elements\n4\n", "$Elements\n2000000000\n")),
    ("missing section '$Nodes'", lambda t: t.replace("$Nodes", "$Nodez").replace("$EndNodez", "$EndNodes")),
    ("missing section '$Elements'", lambda t: t.replace("$Elements", "$Elementz")),
    # the earlier line wins: a dimension error on element 3 before a bad number on element 4
    ("element of dimension 1", lambda t: edit(edit(t, "3 1 2 2 2 1 2", "3 1 2 1 2 1 2"), "4 2 2 3 3 2 3 4",
                                                "4 2 2 3 3 2 x 4")),
    # on one line the region is checked before the node list
    ("element of dimension 1", lambda t: edit(t, "3 1 2 2 2 1 2", "3 1 2 1 2 1 7")),
]


@pytest.mark.parametrize("case", range(len(ERRORS)))
def test_errors_name_the_first_offending_line(tmp_path, case):
    frag, mutate = ERRORS[case]
    p = tmp_path / "e.msh"
    p.write_text(mutate(BASE))
    with pytest.raises(G.GmshError) as r:
        G.read_mesh(str(p))
    with pytest.raises(ValueError) as g:
        mhdarcy.read_gmsh(str(p))
    msg = str(g.value)
    assert frag in msg and frag in str(r.value), (msg, str(r.value))
    m = re.search(r"e\.msh:(\d+):", msg)
    assert (int(m.group(1)) if m else -1) == r.value.line, (msg, r.value.line)


def test_truncated_and_missing_files(tmp_path):
    p = tmp_path / "t.msh"
    p.write_text(BASE[:BASE.index("4 2 2 3")])
    with pytest.raises(ValueError, match="end of file"):
        mhdarcy.read_gmsh(str(p))
    with pytest.raises(OSError, match="cannot open"):
        mhdarcy.read_gmsh(str(tmp_path / "absent.msh"))
    with pytest.raises(OSError, match="cannot open"):
        mhdarcy.read_element_data(str(tmp_path / "absent.msh"), "f", [1])
    ok = tmp_path / "ok.msh"
    ok.write_text(BASE)
    m = mhdarcy.read_gmsh(str(ok))
    assert m.regions == [(1, 2, False, "plane"), (2, 1, True, ".edge"), (3, 2, False, "other")]
    assert list(m.el_id) == [1, 2, 4] and list(m.bc_id) == [3] and list(m.el_region) == [1, 1, 3]


def data_file(rng, ids, fields, n_sections, rows_per_section, junk=True):
    """Random $ElementData sections: ascending row ids drawn from ids and from ids that are
    not elements, times that repeat and decrease, 1 or 3 components."""
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat"]
    for s in range(n_sections):
        f = fields[rng.integers(len(fields))]
        nc = int(rng.choice([1, 3]))
        pool = np.union1d(ids, rng.integers(0, ids.max() + 50, 200) if junk else [])
        rows = np.sort(rng.choice(pool, size=min(rows_per_section, len(pool)), replace=False))
        t = float(rng.choice([0.0, 0.5, 1.0, 2.5]))
        out += ["$ElementData", "1", '"%s"' % f, "1", repr(t), "3", str(s), str(nc), str(len(rows))]
        for r in rows:
            out.append(" ".join([str(int(r))] + ["%.17g" % v for v in rng.normal(size=nc)]))
        out.append("$EndElementData")
    return "\n".join(out) + "\n"


@pytest.mark.parametrize("seed,rows", [(0, 40), (1, 300), (2, 20000)])
def test_element_data_matches_restatement(tmp_path, seed, rows):
    rng = np.random.default_rng(seed)
    ids = np.unique(rng.integers(1, 3 * rows + 10, size=max(rows, 20)))
    p = tmp_path / "d.msh"
    big = rows > 1000
    p.write_text(data_file(rng, ids, ["cond", "aniso", "src"], 4 if big else 6, rows))
    if big:
        assert p.stat().st_size > (1 << 20)
    for field in ("cond", "aniso", "src"):
        for t in ((0.5, 9.0) if big else (0.0, 0.5, 1.0, 2.0, 9.0)):
            for sub in ((ids[::3],) if big else (ids, ids[::4])):
                for nc in (1, 3):
                    try:
                        ref = G.read_element_data(str(p), field, sub, t, nc)
                    except ValueError:
                        with pytest.raises(ValueError):
                            mhdarcy.read_element_data(str(p), field, sub, t, nc)
                        continue
                    got = mhdarcy.read_element_data(str(p), field, sub, t, nc)
                    assert np.array_equal(got, ref, equal_nan=True), (field, t, nc)
