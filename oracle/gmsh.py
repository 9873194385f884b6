"""TEST INFRASTRUCTURE ONLY: a sequential pure-Python restatement of Flow123d's gmsh 2.2 ASCII
input, the checker of the library's parallel reader (mh_gmsh_read, mh_gmsh_element_data).
Never imported by the product; used by tests/ on small files.

It follows the reference step by step:
  * Tokenizer (src/system/tokenizer.cc:54-120): lines are trimmed, empty lines and lines
    starting with '#' are skipped, tokens are separated by blanks with '"' quoting and '\\'
    escapes (boost escaped_list_separator), empty tokens are dropped; skip_to finds the next
    line containing a pattern;
  * GmshMeshReader::read_physical_names / read_nodes / read_elements
    (src/mesh/msh_gmshreader.cc:89-244) with RegionDB::add_region (src/mesh/region.cc:107-175):
    a name starting with '.' marks a boundary region, an id seen only in $Elements becomes the
    bulk region "region_<id>", an element of another dimension than its region is an error,
    elements of boundary regions are boundary elements, points in bulk regions are dropped;
    a repeated node or element id is an error (ElementVector::add_item, sys_vector.hh:371);
  * read_data_header / read_element_data (msh_gmshreader.cc:251-396) for $ElementData.
Errors raise GmshError(line, message), line being the 1-based line of the file.
"""
import math
import re

import numpy as np

TYPES = {1: 1, 2: 2, 4: 3, 15: 0}


class GmshError(ValueError):
    def __init__(self, line, msg):
        self.line = line
        super().__init__(f"line {line}: {msg}")


def tokens(line):
    out, cur, quoted, i = [], [], False, 0
    while i < len(line):
        c = line[i]
        if c == "\\" and i + 1 < len(line):
            i += 1
            cur.append("\n" if line[i] == "n" else line[i])
        elif c == '"':
            quoted = not quoted
        elif not quoted and c in " \t":
            if cur:
                out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
        i += 1
    if cur:
        out.append("".join(cur))
    return out


class Tok:
    """The content lines of a file as (1-based file line, text)."""

    def __init__(self, text):
        self.lines = []
        for n, raw in enumerate(text.split("\n"), 1):
            s = raw.strip(" \t\r\v\f")
            if s and not s.startswith("#"):
                self.lines.append((n, s))

    def line_no(self, k):
        return self.lines[k][0] if k < len(self.lines) else -1

    def toks(self, k):
        if k >= len(self.lines):
            raise GmshError(-1, "unexpected end of file")
        return tokens(self.lines[k][1])

    def skip_to(self, k, pat, stop=None):
        while k < len(self.lines):
            if pat in self.lines[k][1]:
                return k
            if stop is not None and stop in self.lines[k][1]:
                return None
            k += 1
        return None


def _u32(tok, line):
    s = tok[1:] if tok.startswith("+") else tok
    if not s.isdigit() or not s.isascii() or int(s) > 0xFFFFFFFF:
        raise GmshError(line, "wrong format of number")
    return int(s)


_FLOAT = re.compile(r"-?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|[iI][nN][fF](?:[iI][nN][iI][tT][yY])?|"
                    r"[nN][aA][nN](?:\([0-9A-Za-z_]*\))?)")


def _f64(tok, line):
    """std::from_chars (general format) after one optional '+': a result out of range (overflow,
    or underflow to zero) is an error."""
    s = tok[1:] if tok.startswith("+") else tok
    if not _FLOAT.fullmatch(s):
        raise GmshError(line, "wrong format of number")
    v = float(s)
    if math.isinf(v) and "n" not in s.lower():
        raise GmshError(line, "wrong format of number")  # overflow
    if v == 0.0 and re.search(r"[1-9]", re.split(r"[eE]", s)[0]):
        raise GmshError(line, "wrong format of number")  # underflow to zero
    return v


class Stream:
    """Sequential reader of one line's tokens."""

    def __init__(self, tok, k):
        self.t = tok.toks(k)
        self.line = tok.line_no(k)
        self.i = 0

    def next(self):
        if self.i >= len(self.t):
            raise GmshError(self.line, "wrong format of number")
        self.i += 1
        return self.t[self.i - 1]

    def u32(self):
        return _u32(self.next(), self.line)

    def f64(self):
        return _f64(self.next(), self.line)


def read_mesh(path):
    """dict with nodes, node_id, el_* and bc_* arrays in file order, and the region table."""
    tok = Tok(open(path, encoding="latin-1").read())
    regions = []  # (id, dim, boundary, name)
    by_id, by_name = {}, {}

    def add_named(rid, name, dim, line):
        bdr = name.startswith(".")
        if rid in by_id:
            r = regions[by_id[rid]]
            if r[3] != name:
                raise GmshError(line, f"region id {rid} named '{name}' already names '{r[3]}'")
            if r[1] != dim:
                raise GmshError(line, f"region '{name}' given dimensions {r[1]} and {dim}")
            if r[2] != bdr:
                raise GmshError(line, f"region '{name}' is both boundary and bulk")
            return by_id[rid]
        if name in by_name:
            raise GmshError(line, f"region name '{name}' already belongs to id {regions[by_name[name]][0]}")
        by_id[rid] = by_name[name] = len(regions)
        regions.append((rid, dim, bdr, name))
        return len(regions) - 1

    k = tok.skip_to(0, "$PhysicalNames", "$Nodes")
    cur = 0
    if k is not None:
        n = Stream(tok, k + 1).u32()
        for i in range(n):
            s = Stream(tok, k + 2 + i)
            dim, rid = s.u32(), s.u32()
            name = s.t[s.i] if s.i < len(s.t) else ""
            add_named(rid, name, dim, s.line)
        cur = k + 1 + n
    k = tok.skip_to(cur, "$Nodes")
    if k is None:
        raise GmshError(-1, "missing section '$Nodes'")
    nn = Stream(tok, k + 1).u32()
    if nn == 0:
        raise GmshError(tok.line_no(k + 1), "zero number of nodes")
    node_index, node_id, xyz = {}, [], []
    for i in range(nn):
        s = Stream(tok, k + 2 + i)
        nid = s.u32()
        p = [s.f64(), s.f64(), s.f64()]
        if nid in node_index:
            raise GmshError(s.line, f"repeated node id {nid}")
        node_index[nid] = i
        node_id.append(nid)
        xyz.append(p)
    k = tok.skip_to(k + 1 + nn, "$Elements")
    if k is None:
        raise GmshError(-1, "missing section '$Elements'")
    ne = Stream(tok, k + 1).u32()
    if ne == 0:
        raise GmshError(tok.line_no(k + 1), "zero number of elements")
    bulk, bnd = [], []
    seen_bulk, seen_bnd = set(), set()
    for i in range(ne):
        s = Stream(tok, k + 2 + i)
        eid, typ = s.u32(), s.u32()
        if typ not in TYPES:
            raise GmshError(s.line, f"element {eid} is of the unsupported type {typ}")
        dim = TYPES[typ]
        ntags = s.u32()
        if ntags < 2:
            raise GmshError(s.line, f"element {eid} has fewer than two tags")
        rid, _obj = s.u32(), s.u32()
        part = s.u32() if ntags > 2 else 0
        for _ in range(3, ntags):
            s.u32()
        if rid in by_id:
            r = regions[by_id[rid]]
            if r[1] != dim:
                raise GmshError(s.line, f"element {eid}: element of dimension {dim} in region '{r[3]}'")
        else:
            add_named(rid, f"region_{rid}", dim, s.line)
        boundary = regions[by_id[rid]][2]
        if boundary:
            if eid in seen_bnd:
                raise GmshError(s.line, f"repeated boundary element id {eid}")
            seen_bnd.add(eid)
        elif dim > 0:
            if eid in seen_bulk:
                raise GmshError(s.line, f"repeated element id {eid}")
            seen_bulk.add(eid)
        nodes = []
        for _ in range(dim + 1):
            nid = s.u32()
            if nid not in node_index:
                raise GmshError(s.line, f"unknown node id {nid} in element {eid}")
            nodes.append(node_index[nid])
        rec = (eid, dim, nodes + [-1] * (4 - len(nodes)), rid, min(part, 2 ** 31 - 1))
        if boundary:
            bnd.append(rec)
        elif dim > 0:
            bulk.append(rec)
    col = lambda recs, j, dt: np.array([r[j] for r in recs], dt)
    return dict(nodes=np.array(xyz, np.float64).reshape(-1, 3), node_id=np.array(node_id, np.int64),
                el_id=col(bulk, 0, np.int64), el_dim=col(bulk, 1, np.int32),
                el_nodes=col(bulk, 2, np.int32).reshape(-1, 4), el_region=col(bulk, 3, np.int32),
                el_partition=col(bulk, 4, np.int32), bc_id=col(bnd, 0, np.int64), bc_dim=col(bnd, 1, np.int32),
                bc_nodes=col(bnd, 2, np.int32).reshape(-1, 4), bc_region=col(bnd, 3, np.int32),
                regions=regions)


def read_element_data(path, field_name, el_ids, time=0.0, n_components=1):
    """[len(el_ids), n_components] values of the field at `time`, NaN where no section gave
    one (read_element_data, msh_gmshreader.cc:306-396)."""
    ids = [int(v) for v in el_ids]
    if any(b <= a for a, b in zip(ids, ids[1:])):
        raise ValueError("el_ids must be strictly ascending")
    tok = Tok(open(path, encoding="latin-1").read())
    out = np.full((len(ids), n_components), np.nan)
    limit = time * (1.0 + 2.0 * np.finfo(float).eps)
    found = used = False
    k = 0
    while True:
        k = tok.skip_to(k, "$ElementData")
        if k is None:
            break
        h = k + 1
        n_str = Stream(tok, h).u32()
        name = ""
        if n_str:
            h += 1
            t = tok.toks(h)
            name = t[0] if t else ""
            h += n_str - 1
        h += 1
        n_real = Stream(tok, h).u32()
        t_sec = 0.0
        if n_real:
            h += 1
            t_sec = Stream(tok, h).f64()
            h += n_real - 1
        h += 1
        n_int = Stream(tok, h).u32()
        ints = [0, 1, 0]
        for j in range(min(n_int, 3)):
            h += 1
            ints[j] = Stream(tok, h).u32()
        h += max(n_int - 3, 0)
        k = h + 1
        if name != field_name:
            continue
        found = True
        if t_sec > limit:
            break
        used = True
        n_ent = ints[2]
        pos = 0
        for r in range(n_ent):
            if k + r >= len(tok.lines):
                break
            s = Stream(tok, k + r)
            eid = s.u32()
            while pos < len(ids) and ids[pos] < eid:
                pos += 1
            if pos == len(ids):
                break
            if ids[pos] == eid:
                try:
                    out[pos] = [s.f64() for _ in range(n_components)]
                except GmshError:
                    raise GmshError(s.line, f"element {eid} of field '{field_name}' has fewer than "
                                            f"{n_components} values or a malformed one")
        k += n_ent
    if not found:
        raise ValueError(f"{path}: no $ElementData section for field '{field_name}'")
    if not used:
        raise ValueError(f"{path}: no $ElementData of field '{field_name}' at or before time {time}")
    return out
