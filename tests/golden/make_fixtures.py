"""Generates the golden fixtures under tests/golden/ from the Flow123d reference tree.

Run once where the reference sources are available, giving the root of their tree:
    python tests/golden/make_fixtures.py REFERENCE_ROOT
Each case is written as <case>.npz holding the mesh (nodes, bulk and boundary elements with
their physical regions), the coefficient and boundary data of the case's .con file (evaluated
the way the reference evaluates them: element fields per region, boundary fields at the
boundary element's barycentre, bc_piezo_head converted to pressure by adding the potential
(0,0,-1).x as FieldAddPotential does), and the reference's own results:
  * t01            tests/01_steady_flow_123d (flow_gmsh.con): ref_output raw_output.txt, i.e.
                   per element pressure, barycentric flux, side (edge) pressures, side fluxes;
                   the node pressures of the output mesh ($NodeData "pressure_nodes_[L]"); the
                   boundary and source tables of water_balance.out;
  * t02            tests/02_transport_12d (flow part of flow_gmsh.con): legacy side-based Dirichlet
                   data on a 1D-2D network; element and node pressures, element velocities and
                   the water balance;
  * t03            tests/03_transport_small_12d (flow part of flow_vtk.con): element and node
                   pressures, element velocities of the VTK output and the water balance of a
                   1D-2D network with a three-channel junction;
  * t05_*          tests/05_flow_boundary_conditions: element pressures of the VTK output and the
                   water balance;
  * t08            tests/08_steady_flow_sources: element and node pressures, element velocities
                   of the VTK output, and its water balance (a source field given by a formula);
  * t06_32, t06_21 tests/06_flow_coupling: element pressures of the VTK output and the water balance;
  * t10_mh         tests/10_unsteady_2d (flow_MH.con): element pressures at t = 0.1 .. 0.5;
  * t10_lmh        the same with the lumped scheme (flow_LMH.con);
  * t13            tests/13_edge_solute_mixing: legacy side-based boundary data, the flow outputs
                   and the concentrations of the explicit transport every 0.5 up to t = 100;
  * t14            tests/14_trans_time_bc (trans_explicit.con): an inflow concentration switched
                   in time by four legacy transport files; concentrations every 1.0 up to t = 10.
The parsers here are self-contained (independent of the package under test).
"""
import os
import re
import sys

import numpy as np

if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], "tests")):
    sys.exit("usage: make_fixtures.py REFERENCE_ROOT  (the Flow123d source tree, holding tests/)")
REF = sys.argv[1]
OUT = os.path.dirname(os.path.abspath(__file__))
TDIM = {1: 1, 2: 2, 4: 3, 15: 0}


def parse_gmsh(path):
    txt = open(path).read().split("\n")
    names, node_ids, xyz, elems = {}, [], [], []
    i = 0
    while i < len(txt):
        t = txt[i].strip()
        if t == "$PhysicalNames":
            n = int(txt[i + 1])
            for k in range(n):
                d, rid, nm = txt[i + 2 + k].split(None, 2)
                names[int(rid)] = nm.strip().strip('"')
            i += n + 2
        elif t == "$Nodes":
            n = int(txt[i + 1])
            for k in range(n):
                p = txt[i + 2 + k].split()
                node_ids.append(int(p[0]))
                xyz.append([float(v) for v in p[1:4]])
            i += n + 2
        elif t == "$Elements":
            n = int(txt[i + 1])
            for k in range(n):
                p = [int(v) for v in txt[i + 2 + k].split()]
                elems.append(p)
            i += n + 2
        else:
            i += 1
    nmap = {nid: k for k, nid in enumerate(node_ids)}
    bulk, bnd = [], []
    for p in elems:
        eid, et, nt = p[0], p[1], p[2]
        d = TDIM[et]
        reg = p[3]
        nd = [nmap[v] for v in p[3 + nt:3 + nt + d + 1]] + [-1] * (3 - d)
        if names.get(reg, "").startswith("."):
            bnd.append((eid, d, nd, reg))
        elif d > 0:
            bulk.append((eid, d, nd, reg))
    return dict(
        nodes=np.array(xyz), el_id=np.array([b[0] for b in bulk]), el_dim=np.array([b[1] for b in bulk], np.int32),
        el_nodes=np.array([b[2] for b in bulk], np.int32), el_region=np.array([b[3] for b in bulk], np.int32),
        bc_id=np.array([b[0] for b in bnd]), bc_dim=np.array([b[1] for b in bnd], np.int32),
        bc_nodes=np.array([b[2] for b in bnd], np.int32).reshape(-1, 4),
        bc_region=np.array([b[3] for b in bnd], np.int32)), names


def centres(nodes, dims, conn):
    out = np.zeros((len(dims), 3))
    for k, (d, c) in enumerate(zip(dims, conn)):
        out[k] = nodes[c[:d + 1]].mean(axis=0)
    return out


def vtu_cell_array(path, name):
    txt = open(path).read()
    m = re.search(r'<DataArray[^>]*Name="' + re.escape(name) + r'"[^>]*>(.*?)</DataArray>', txt, re.S)
    return np.array([float(v) for v in m.group(1).split()])


def raw_output(path):
    lines = open(path).read().split("\n")
    k = next(i for i, l in enumerate(lines) if l.startswith("$FlowField"))
    n = int(lines[k + 2])
    ids, p, flux, ns, sp, sf = [], [], [], [], np.zeros((n, 4)), np.zeros((n, 4))
    for j in range(n):
        v = lines[k + 3 + j].split()
        ids.append(int(v[0]))
        p.append(float(v[1]))
        flux.append([float(x) for x in v[2:5]])
        m = int(v[5])
        ns.append(m)
        sp[j, :m] = [float(x) for x in v[6:6 + m]]
        sf[j, :m] = [float(x) for x in v[6 + m:6 + 2 * m]]
    return dict(ref_el_id=np.array(ids), ref_pressure=np.array(p), ref_flux=np.array(flux),
                ref_n_sides=np.array(ns, np.int32), ref_side_pressure=sp, ref_side_flux=sf)


def gmsh_node_data(path, name, mesh_path):
    """Values of the $NodeData block `name` of an output mesh, ordered as the nodes of the
    input mesh (matched by node id)."""
    txt = open(path).read().split("\n")
    k = next(i for i, l in enumerate(txt) if l.strip() == "$NodeData" and txt[i + 2].strip().strip('"') == name)
    n_str = int(txt[k + 1])
    n_real = int(txt[k + 2 + n_str])
    n_int = int(txt[k + 3 + n_str + n_real])
    first = k + 4 + n_str + n_real + n_int
    vals = {}
    for line in txt[first:]:
        if line.startswith("$EndNodeData"):
            break
        nid, v = line.split()[:2]
        vals[int(nid)] = float(v)
    mtxt = open(mesh_path).read().split("\n")
    j = next(i for i, l in enumerate(mtxt) if l.strip() == "$Nodes")
    ids = [int(mtxt[j + 2 + q].split()[0]) for q in range(int(mtxt[j + 1]))]
    return np.array([vals[i] for i in ids])


def water_balance(path):
    """The boundary table (region id, total, outflow, inflow) and the source table (region id,
    total) of a water_balance.out."""
    bdr, src, mode = [], [], None
    for line in open(path).read().split("\n"):
        if line.startswith("# Boundary water balance"):
            mode = "b"
        elif line.startswith("# Source fluxes"):
            mode = "s"
        elif line.startswith("#") or not line.strip():
            continue
        elif mode == "b":  # id, label (may hold blanks), total, outflow, inflow, time
            v = line.split()
            bdr.append([float(v[0]), float(v[-4]), float(v[-3]), float(v[-2])])
        elif mode == "s":  # id, label, total, time
            v = line.split()
            src.append([float(v[0]), float(v[-2])])
    return dict(ref_bdr_balance=np.array(bdr), ref_src_balance=np.array(src))


def case(mesh_path, bulk, bcs, extra, out_name, meta):
    m, names = parse_gmsh(mesh_path)
    rid = {v: k for k, v in names.items()}
    ne, nb = len(m["el_dim"]), len(m["bc_dim"])
    f = dict(conductivity=np.ones(ne), anisotropy=np.ones(ne), cross_section=np.ones(ne), sigma=np.ones(ne),
             water_source_density=np.zeros(ne), storativity=np.ones(ne), init_pressure=np.zeros(ne))
    el_c = centres(m["nodes"], m["el_dim"], m["el_nodes"])
    for reg, vals in bulk.items():
        sel = m["el_region"] == rid[reg]
        assert sel.any(), reg
        for k, v in vals.items():
            # a formula field is evaluated at the element centre, as the assembly does
            f[k][sel] = [v(*c) for c in el_c[sel]] if callable(v) else v
    bc_c = centres(m["nodes"], m["bc_dim"], m["bc_nodes"])
    b = dict(bc_type=np.zeros(nb, np.int32), bc_pressure=np.zeros(nb), bc_flux=np.zeros(nb),
             bc_robin_sigma=np.zeros(nb))
    types = {"none": 0, "dirichlet": 1, "neumann": 2, "robin": 3}
    for reg, spec in bcs.items():
        sel = np.where(m["bc_region"] == rid[reg])[0]
        assert len(sel), reg
        b["bc_type"][sel] = types[spec["type"]]
        for key in ("pressure", "flux", "robin_sigma"):
            if key in spec:
                b["bc_" + key][sel] = [spec[key](*bc_c[i]) for i in sel]
        if "piezo_head" in spec:  # FieldAddPotential with gravity (0,0,-1,0): p = h - z
            b["bc_pressure"][sel] = [spec["piezo_head"](*bc_c[i]) - bc_c[i][2] for i in sel]
    np.savez_compressed(os.path.join(OUT, out_name + ".npz"), **m, **f, **b, **extra,
                        meta=np.array(meta))
    print(out_name, ne, "elements", nb, "boundary elements", list(extra))


def legacy_flow_bcd(path):
    """Rows of a legacy flow boundary file ($BoundaryConditions): (condition id, type, value,
    element id, local side) for conditions given by element and side (OldBcdInput::read_flow,
    src/flow/old_bcd.cc): type 1 Dirichlet (value = pressure), 2 Neumann (value = flux)."""
    lines = open(path).read().split("\n")
    k = next(i for i, l in enumerate(lines) if l.strip() == "$BoundaryConditions")
    rows = []
    for line in lines[k + 2:k + 2 + int(lines[k + 1])]:
        v = line.split()
        cid, typ = int(v[0]), int(v[1])
        assert typ in (1, 2) and int(v[3]) == 2, line  # value, then "by element and side"
        rows.append((cid, typ, float(v[2]), int(v[4]), int(v[5])))
    return rows


def legacy_transport_bcd(path):
    """{condition id: concentrations} of a legacy transport boundary file ($Transport_BCD):
    each row names the flow condition whose boundary it applies to (OldBcdInput::read_transport)."""
    lines = open(path).read().split("\n")
    k = next(i for i, l in enumerate(lines) if l.strip() == "$Transport_BCD")
    out = {}
    for line in lines[k + 2:k + 2 + int(lines[k + 1])]:
        v = line.split()
        out[int(v[0])] = [float(x) for x in v[2:]]
    return out


def gmsh_element_data_blocks(path, name):
    """(times, values [n_blocks, n_entities]) of every $ElementData block of a field, in file order."""
    txt = open(path).read().split("\n")
    times, vals = [], []
    for k, l in enumerate(txt):
        if l.strip() != "$ElementData" or txt[k + 2].strip().strip('"') != name:
            continue
        n_str = int(txt[k + 1])
        n_real = int(txt[k + 2 + n_str])
        times.append(float(txt[k + 3 + n_str]) if n_real else 0.0)
        n_int = int(txt[k + 3 + n_str + n_real])
        n_ent = int(txt[k + 6 + n_str + n_real])
        first = k + 4 + n_str + n_real + n_int
        vals.append([float(r.split()[1]) for r in txt[first:first + n_ent]])
    return np.array(times), np.array(vals)


def case_t13(t):
    """tests/13_edge_solute_mixing (flow_gmsh.con): a fork of three strips meeting on one edge,
    flow and transport boundary conditions in the legacy side-based files, explicit convection of
    one substance up to t = 100 with output every 0.5."""
    d = lambda *p: t("13_edge_solute_mixing", *p)
    m, names = parse_gmsh(d("input", "test13.msh"))
    ne = len(m["el_dim"])
    aniso = {17: 1.0, 18: 0.1, 19: 1.0}
    f = dict(conductivity=np.ones(ne), anisotropy=np.array([aniso[r] for r in m["el_region"]]),
             cross_section=np.ones(ne), sigma=np.ones(ne), water_source_density=np.zeros(ne),
             storativity=np.ones(ne), init_pressure=np.zeros(ne))
    fb = legacy_flow_bcd(d("input", "test13.fbc"))
    tb = legacy_transport_bcd(d("input", "test13.tbc"))
    eidx = {int(e): i for i, e in enumerate(m["el_id"])}
    legacy = dict(lbc_id=np.array([r[0] for r in fb], np.int32), lbc_type=np.array([r[1] for r in fb], np.int32),
                  lbc_value=np.array([r[2] for r in fb]), lbc_element=np.array([eidx[r[3]] for r in fb], np.int32),
                  lbc_side=np.array([r[4] for r in fb], np.int32),
                  lbc_conc=np.array([tb.get(r[0], [0.0])[0] for r in fb]))
    out = d("ref_output", "flow_gmsh.con")
    ct, cv = gmsh_element_data_blocks(os.path.join(out, "transport.msh"), "A_mobile_[M/L^3]")
    fl = os.path.join(out, "test13.msh")
    ref = dict(ref_pressure=gmsh_element_data_blocks(fl, "pressure_elements_[L]")[1][0],
               ref_flux=np.array(gmsh_element_vectors(fl, "velocity_elements_[L/T]")),
               ref_node_pressure=gmsh_node_data(fl, "pressure_nodes_[L]", d("input", "test13.msh")),
               ref_conc_times=ct, ref_conc=cv)
    np.savez_compressed(os.path.join(OUT, "t13.npz"), **m, **f, **legacy, **ref,
                        meta=np.array("tests/13_edge_solute_mixing flow_gmsh.con: legacy .fbc/.tbc boundary "
                                      "data, transport.msh concentrations every 0.5 (por_m = 1), flow outputs"))
    print("t13", ne, "elements", len(fb), "legacy conditions", len(ct), "concentration outputs")


def case_t02(t):
    """tests/02_transport_12d (flow part of flow_gmsh.con): a 1D network (anisotropy 10) on the
    edges of a 2D domain, Dirichlet conditions in the legacy side-based file, solver r_tol 1e-12;
    the flow outputs of test2.msh (printed with 6 digits) and its water balance."""
    d = lambda *p: t("02_transport_12d", *p)
    m, names = parse_gmsh(d("input", "test2.msh"))
    ne = len(m["el_dim"])
    aniso = {48: 10.0, 184: 1.0}
    f = dict(conductivity=np.ones(ne), anisotropy=np.array([aniso[r] for r in m["el_region"]]),
             cross_section=np.ones(ne), sigma=np.ones(ne), water_source_density=np.zeros(ne),
             storativity=np.ones(ne), init_pressure=np.zeros(ne))
    fb = legacy_flow_bcd(d("input", "test2.fbc"))
    eidx = {int(e): i for i, e in enumerate(m["el_id"])}
    legacy = dict(lbc_id=np.array([r[0] for r in fb], np.int32), lbc_type=np.array([r[1] for r in fb], np.int32),
                  lbc_value=np.array([r[2] for r in fb]), lbc_element=np.array([eidx[r[3]] for r in fb], np.int32),
                  lbc_side=np.array([r[4] for r in fb], np.int32), lbc_conc=np.zeros(len(fb)))
    out = d("ref_output", "flow_gmsh.con")
    fl = os.path.join(out, "test2.msh")
    ref = dict(ref_pressure=gmsh_element_data_blocks(fl, "pressure_elements_[L]")[1][0],
               ref_flux=np.array(gmsh_element_vectors(fl, "velocity_elements_[L/T]")),
               ref_node_pressure=gmsh_node_data(fl, "pressure_nodes_[L]", d("input", "test2.msh")),
               **water_balance(os.path.join(out, "water_balance.txt")))
    np.savez_compressed(os.path.join(OUT, "t02.npz"), **m, **f, **legacy, **ref,
                        meta=np.array("tests/02_transport_12d flow_gmsh.con: legacy .fbc boundary data, flow "
                                      "outputs of test2.msh (6 digits), water_balance.txt; r_tol 1e-12"))
    print("t02", ne, "elements", len(fb), "legacy conditions")


def case_t14(t):
    """tests/14_trans_time_bc (trans_explicit.con): a strip with a uniform flow, Dirichlet
    pressures in the legacy side-based file, and the inflow concentration switched by four legacy
    transport files at t = 1 (20), 3 (0), 6 (40) and 7 (0), 0 before; explicit convection up to
    t = 10 with output every 1.0 (VTK, 16 digits)."""
    d = lambda *p: t("14_trans_time_bc", *p)
    m, names = parse_gmsh(d("input", "test14.msh"))
    ne = len(m["el_dim"])
    f = dict(conductivity=np.ones(ne), anisotropy=np.full(ne, 0.1), cross_section=np.ones(ne), sigma=np.ones(ne),
             water_source_density=np.zeros(ne), storativity=np.ones(ne), init_pressure=np.zeros(ne))
    fb = legacy_flow_bcd(d("input", "test14.fbc"))
    eidx = {int(e): i for i, e in enumerate(m["el_id"])}
    times = [1.0, 3.0, 6.0, 7.0]
    tb = [legacy_transport_bcd(d("input", "test14_tbc_%03d" % k)) for k in range(4)]
    legacy = dict(lbc_id=np.array([r[0] for r in fb], np.int32), lbc_type=np.array([r[1] for r in fb], np.int32),
                  lbc_value=np.array([r[2] for r in fb]), lbc_element=np.array([eidx[r[3]] for r in fb], np.int32),
                  lbc_side=np.array([r[4] for r in fb], np.int32),
                  lbc_conc_times=np.array(times),
                  lbc_conc_steps=np.array([[b.get(r[0], [0.0])[0] for r in fb] for b in tb]))
    out = d("ref_output", "trans_explicit.con")
    vt = lambda k: vtu_cell_array(os.path.join(out, "transport", "transport-%06d.vtu" % k), "A_mobile_[M/L^3]")
    fl = os.path.join(out, "test14", "test14-000000.vtu")
    ref = dict(ref_pressure=vtu_cell_array(fl, "pressure_elements_[L]"),
               ref_flux=vtu_cell_array(fl, "velocity_elements_[L/T]").reshape(-1, 3),
               ref_conc_times=np.arange(11.0), ref_conc=np.array([vt(k) for k in range(11)]))
    np.savez_compressed(os.path.join(OUT, "t14.npz"), **m, **f, **legacy, **ref,
                        meta=np.array("tests/14_trans_time_bc trans_explicit.con: legacy .fbc and four time-switched "
                                      "transport files, VTK concentrations every 1.0 up to t = 10"))
    print("t14", ne, "elements", len(fb), "legacy conditions")


def gmsh_element_vectors(path, name):
    """The first $ElementData block of a 3-component field: [n_entities, 3]."""
    txt = open(path).read().split("\n")
    k = next(i for i, l in enumerate(txt) if l.strip() == "$ElementData" and txt[i + 2].strip().strip('"') == name)
    n_str = int(txt[k + 1])
    n_real = int(txt[k + 2 + n_str])
    n_int = int(txt[k + 3 + n_str + n_real])
    n_ent = int(txt[k + 6 + n_str + n_real])
    first = k + 4 + n_str + n_real + n_int
    return [[float(x) for x in r.split()[1:4]] for r in txt[first:first + n_ent]]


def main():
    t = lambda *p: os.path.join(REF, "tests", *p)
    # test 01: 1D-2D-3D steady flow, n_schurs = 2
    case(t("01_steady_flow_123d", "input", "test1_new.msh"),
         {"1d_channel": {"anisotropy": 10.0}, "2d_fraction_1": {"anisotropy": 1.0},
          "2d_fraction_2": {"anisotropy": 1.0}, "3d_cube": {"anisotropy": 0.1}},
         {r: {"type": "dirichlet", "pressure": lambda x, y, z: x - z}
          for r in (".1d_channel", ".2d_fraction_1", ".2d_fraction_2", ".3d_cube")},
         {**raw_output(t("01_steady_flow_123d", "ref_output", "flow_gmsh.con", "raw_output.txt")),
          "ref_node_pressure": gmsh_node_data(t("01_steady_flow_123d", "ref_output", "flow_gmsh.con", "test1.msh"),
                                              "pressure_nodes_[L]", t("01_steady_flow_123d", "input",
                                                                      "test1_new.msh")),
          **water_balance(t("01_steady_flow_123d", "ref_output", "flow_gmsh.con", "water_balance.out"))},
         "t01", "tests/01_steady_flow_123d flow_gmsh.con; raw_output %.8g, node pressures of the output "
         "mesh (%g), water_balance.out (%g); solver -ksp_rtol 1e-10")
    # test 08: sources on a square, exact p = (1-x^2)(1-y^2), homogeneous Dirichlet
    vtu8 = lambda nm: vtu_cell_array(t("08_steady_flow_sources", "ref_output", "flow_vtk.con", "flow",
                                       "flow-000000.vtu"), nm)
    case(t("08_steady_flow_sources", "input", "test08.msh"),
         {"plane": {"anisotropy": 1.0,
                    "water_source_density": lambda x, y, z: 2 * (1 - x ** 2) + 2 * (1 - y ** 2)}},
         {".plane_boundary": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0}},
         {"ref_pressure": vtu8("pressure_elements_[L]"), "ref_node_pressure": vtu8("pressure_nodes_[L]"),
          "ref_flux": vtu8("velocity_elements_[L/T]").reshape(-1, 3),
          **water_balance(t("08_steady_flow_sources", "ref_output", "flow_vtk.con", "water_balance.txt"))},
         "t08", "tests/08_steady_flow_sources flow_vtk.con VTK (ascii) and water_balance.txt; solver accuracy 1e-7")
    # test 03 (flow part of flow_vtk.con): 1D channels on edges of a 2D square meeting at a
    # junction of three channels, Dirichlet p = x + y on every boundary region (points and lines)
    vtu3 = lambda nm: vtu_cell_array(t("03_transport_small_12d", "ref_output", "flow_vtk.con", "test3",
                                       "test3-000000.vtu"), nm)
    case(t("03_transport_small_12d", "input", "mesh_with_boundary.msh"),
         {"1d_upper": {"conductivity": 10.0}, "1d_lower": {"conductivity": 10.0},
          "1d_left_branch": {"conductivity": 10.0}, "2d": {"conductivity": 1.0}},
         {r: {"type": "dirichlet", "pressure": lambda x, y, z: x + y}
          for r in (".1d_top", ".1d_left", ".1d_bottom", ".2d_top", ".2d_right", ".2d_bottom", ".2d_left")},
         {"ref_pressure": vtu3("pressure_elements_[L]"), "ref_node_pressure": vtu3("pressure_nodes_[L]"),
          "ref_flux": vtu3("velocity_elements_[L/T]").reshape(-1, 3),
          **water_balance(t("03_transport_small_12d", "ref_output", "flow_vtk.con", "water_balance.txt"))},
         "t03", "tests/03_transport_small_12d flow_vtk.con VTK (ascii, 16 digits) and water_balance.txt (%g); "
         "solver r_tol 1e-12, a_tol 1e-12")
    case_t13(t)
    case_t02(t)
    case_t14(t)
    # test 05: Dirichlet / Neumann / Robin on a square, exact u = xy
    vtu5 = lambda c: vtu_cell_array(t("05_flow_boundary_conditions", "ref_output", c, "test05",
                                      "test05-000000.vtu"), "pressure_elements_[L]")
    case(t("05_flow_boundary_conditions", "input", "test05.msh"), {"plane": {"anisotropy": 1.0}},
         {".bc_south": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0},
          ".bc_east": {"type": "dirichlet", "pressure": lambda x, y, z: y},
          ".bc_north": {"type": "dirichlet", "pressure": lambda x, y, z: x},
          ".bc_west": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0}},
         {"ref_pressure": vtu5("flow_dirichlet.con"), **water_balance(t("05_flow_boundary_conditions", "ref_output", "flow_dirichlet.con", "water_balance.out"))}, "t05_dirichlet", "tests/05 flow_dirichlet.con VTK")
    case(t("05_flow_boundary_conditions", "input", "test05.msh"), {"plane": {"anisotropy": 1.0}},
         {".bc_south": {"type": "neumann", "flux": lambda x, y, z: x},
          ".bc_east": {"type": "dirichlet", "pressure": lambda x, y, z: y},
          ".bc_north": {"type": "neumann", "flux": lambda x, y, z: -x},
          ".bc_west": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0}},
         {"ref_pressure": vtu5("flow_neumann.con"), **water_balance(t("05_flow_boundary_conditions", "ref_output", "flow_neumann.con", "water_balance.out"))}, "t05_neumann", "tests/05 flow_neumann.con VTK")
    case(t("05_flow_boundary_conditions", "input", "test05.msh"), {"plane": {"anisotropy": 1.0}},
         {".bc_south": {"type": "robin", "pressure": lambda x, y, z: -2 * x, "robin_sigma": lambda x, y, z: 0.5},
          ".bc_east": {"type": "dirichlet", "pressure": lambda x, y, z: y},
          ".bc_north": {"type": "robin", "pressure": lambda x, y, z: 3 * x, "robin_sigma": lambda x, y, z: 0.5},
          ".bc_west": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0}},
         {"ref_pressure": vtu5("flow_robin.con"), **water_balance(t("05_flow_boundary_conditions", "ref_output", "flow_robin.con", "water_balance.out"))}, "t05_robin", "tests/05 flow_robin.con VTK")
    # test 06: dimension coupling, known answers p2 = -3 (head), p1 = -2.5
    case(t("06_flow_coupling", "input", "test6_32d.msh"),
         {"2d_fraction": {"conductivity": 16.0, "sigma": 1.0, "cross_section": 10.0,
                          "water_source_density": -2.0 / 10.0},
          "3d_cube": {"conductivity": 2.0}},
         {".2d_fraction": {"type": "neumann", "flux": lambda x, y, z: 0.0},
          ".3d_cube": {"type": "dirichlet", "piezo_head": lambda x, y, z: z}},
         {"ref_pressure": vtu_cell_array(t("06_flow_coupling", "ref_output", "flow_32d.con", "test6_32d",
                                           "test6_32d-000000.vtu"), "pressure_elements_[L]"),
          **water_balance(t("06_flow_coupling", "ref_output", "flow_32d.con", "water_balance.out"))},
         "t06_32", "tests/06 flow_32d.con VTK; analytic 2D piezometric head -3")
    case(t("06_flow_coupling", "input", "test6_21d.msh"),
         {"plane": {"conductivity": 5.0, "cross_section": 10.0},
          "channel": {"conductivity": 50.0, "cross_section": 20.0, "sigma": 2.0,
                      "water_source_density": -1.0 / 20.0 * (10.0 * 5.0)}},
         {".plane": {"type": "dirichlet", "piezo_head": lambda x, y, z: x},
          ".channel": {"type": "neumann", "flux": lambda x, y, z: 0.0}},
         {"ref_pressure": vtu_cell_array(t("06_flow_coupling", "ref_output", "flow_21d.con", "test6_21d",
                                           "test6_21d-000000.vtu"), "pressure_elements_[L]"),
          **water_balance(t("06_flow_coupling", "ref_output", "flow_21d.con", "water_balance.out"))},
         "t06_21", "tests/06 flow_21d.con VTK; analytic 1D pressure -2.5")
    # test 10: unsteady MH, dt = 0.01, outputs every 0.1 up to 0.5
    steps = [vtu_cell_array(t("10_unsteady_2d", "ref_output", "flow_MH.con", "test10", "test10-%06d.vtu" % k),
                            "pressure_elements_[L]") for k in range(6)]
    case(t("10_unsteady_2d", "input", "test10.msh"),
         {"plane": {"anisotropy": 0.02, "storativity": 1.0, "init_pressure": 0.0}},
         {".bc_inflow": {"type": "dirichlet", "pressure": lambda x, y, z: 100.0},
          ".bc_outflow": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0}},
         {"ref_pressure_steps": np.array(steps), "ref_times": np.arange(6) * 0.1, "dt": np.array(0.01)},
         "t10_mh", "tests/10_unsteady_2d flow_MH.con VTK every 0.1")
    # the same problem with the lumped mixed-hybrid scheme (Unsteady_LMH)
    steps = [vtu_cell_array(t("10_unsteady_2d", "ref_output", "flow_LMH.con", "test10", "test10-%06d.vtu" % k),
                            "pressure_elements_[L]") for k in range(6)]
    case(t("10_unsteady_2d", "input", "test10.msh"),
         {"plane": {"anisotropy": 0.02, "storativity": 1.0, "init_pressure": 0.0}},
         {".bc_inflow": {"type": "dirichlet", "pressure": lambda x, y, z: 100.0},
          ".bc_outflow": {"type": "dirichlet", "pressure": lambda x, y, z: 0.0}},
         {"ref_pressure_steps": np.array(steps), "ref_times": np.arange(6) * 0.1, "dt": np.array(0.01)},
         "t10_lmh", "tests/10_unsteady_2d flow_LMH.con VTK every 0.1")


if __name__ == "__main__":
    main()
