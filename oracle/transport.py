"""TEST INFRASTRUCTURE ONLY: a pure-Python restatement of the convection matrix of Flow123d's
explicit finite-volume transport, the checker of mh_transport_matrix.  Never imported by the
product; used by tests/ on small meshes (the loops are per element).

ConvectionTransport::create_transport_matrix_mpi (src/transport/transport.cc:788-923), in the
reference's order: for each element i, V_i = |E_i| * cross_section_i * porosity_i,
  * for each side of i that is not on a boundary object: for every other side s of its edge,
    a_{i, el(s)} = -(q_i q_s / (Q_edge |E_i| delta_i por_i)) when q_s > 0 and q_i < 0, else 0,
    Q_edge the sum of the positive side fluxes of the edge (transport.cc:813-820, 840-856);
  * every side with q > 0 (boundary or not) adds -q / V_i to the diagonal (:857-864);
  * for each VB neighbour n of i (i the lower-dimensional element, q the flux of the
    higher-dimensional element's side): a_{i, el2} = q / V_i when q > 0, else 0; when q < 0
    the diagonal of i gets -(-q) / V_i and a_{el2, i} = -q / V_el2, else 0 (:867-890);
  * the diagonal is written last; cfl_max_step = 1 / max_i |a_ii| (:893-906).
MatSetValue(INSERT_VALUES) semantics: a later write of the same entry replaces the earlier one.
"""
import numpy as np
import scipy.sparse as sp


def element_measure(xyz, nodes, dim):
    X = xyz[nodes[:dim + 1]]
    if dim == 1:
        return float(np.linalg.norm(X[1] - X[0]))
    if dim == 2:
        return float(np.linalg.norm(np.cross(X[1] - X[0], X[2] - X[0])) / 2.0)
    return float(abs(np.dot(np.cross(X[1] - X[0], X[2] - X[0]), X[3] - X[0])) / 6.0)


def transport_matrix(mesh, topo, sol, cross_section=1.0, porosity=1.0):
    """(CSR matrix [n_el, n_el] with the reference's entries, cfl_max_step)."""
    xyz = np.asarray(mesh.nodes, np.float64)
    eln = np.asarray(mesh.el_nodes)
    dim = np.asarray(mesh.el_dim)
    ne = len(dim)
    cs = np.broadcast_to(np.asarray(cross_section, np.float64), (ne,))
    por = np.broadcast_to(np.asarray(porosity, np.float64), (ne,))
    ss, se, sb = topo["el_side_start"], topo["side_edge"], topo["side_bdr"]
    n_sides = int(ss[-1])
    side_el = np.repeat(np.arange(ne), np.diff(ss))
    edge_sides = {}
    for s in range(n_sides):
        edge_sides.setdefault(int(se[s]), []).append(s)
    edge_flow = {e: sum(sol[s] for s in sides if sol[s] > 0) for e, sides in edge_sides.items()}
    # VB neighbours of each lower-dimensional element, in creation order
    ngh_el, ngh_side = np.asarray(topo["ngh_element"]), np.asarray(topo["ngh_side"])
    vb = {}
    for n in range(len(ngh_el)):
        vb.setdefault(int(ngh_el[n]), []).append(int(ngh_side[n]))
    meas = np.array([element_measure(xyz, eln[e], dim[e]) for e in range(ne)])
    entries = {}
    max_sum = 0.0
    for i in range(ne):
        aii = 0.0
        for si in range(ss[i], ss[i + 1]):
            flux = sol[si]
            if sb[si] < 0:
                ef = edge_flow[int(se[si])]
                for s in edge_sides[int(se[si])]:
                    if s == si:
                        continue
                    flux2 = sol[s]
                    if flux2 > 0.0 and flux < 0.0:
                        aij = -(flux * flux2 / (ef * meas[i] * cs[i] * por[i]))
                    else:
                        aij = 0.0
                    entries[(i, int(side_el[s]))] = aij
            if flux > 0.0:
                aii -= flux / (meas[i] * cs[i] * por[i])
        for hs in vb.get(i, []):
            el2 = int(side_el[hs])
            flux = sol[hs]
            entries[(i, el2)] = flux / (meas[i] * cs[i] * por[i]) if flux > 0.0 else 0.0
            if flux < 0.0:
                aii -= (-flux) / (meas[i] * cs[i] * por[i])
                aij = (-flux) / (meas[el2] * cs[el2] * por[el2])
            else:
                aij = 0.0
            entries[(el2, i)] = aij
        entries[(i, i)] = aii
        max_sum = max(max_sum, abs(aii))
    keys = sorted(entries)
    rows = np.array([k[0] for k in keys])
    cols = np.array([k[1] for k in keys])
    vals = np.array([entries[k] for k in keys])
    return sp.csr_matrix((vals, (rows, cols)), shape=(ne, ne)), (1.0 / max_sum if max_sum > 0 else np.inf)


def boundary_inflow(mesh, topo, sol, bdr_conc, cross_section=1.0, porosity=1.0):
    """The boundary term of the explicit step (ConvectionTransport::set_boundary_conditions,
    transport.cc:455-491): for every boundary side of element i with inflow (q < 0),
    -q / (|E_i| delta_i por_i) * c_b, c_b the concentration of that boundary object."""
    xyz = np.asarray(mesh.nodes, np.float64)
    eln = np.asarray(mesh.el_nodes)
    dim = np.asarray(mesh.el_dim)
    ne = len(dim)
    cs = np.broadcast_to(np.asarray(cross_section, np.float64), (ne,))
    por = np.broadcast_to(np.asarray(porosity, np.float64), (ne,))
    ss, sb = topo["el_side_start"], topo["side_bdr"]
    out = np.zeros(ne)
    for i in range(ne):
        for s in range(ss[i], ss[i + 1]):
            if sb[s] >= 0 and sol[s] < 0.0:
                out[i] += bdr_conc[sb[s]] * (-(sol[s] / (element_measure(xyz, eln[i], dim[i]) * cs[i] * por[i])))
    return out


def step_count(full_step, cfl):
    """Steps of the time governor over a fixed interval (TimeGovernor::estimate_dt,
    src/coupling/time_governor.cc:261-300): the step is min(interval, CFL step), the count the
    ceiling of interval / step, or its floor when that is within 1e-14 of the ratio."""
    est = min(full_step, cfl)
    ratio = full_step / est
    n = int(np.ceil(ratio))
    nf = int(np.floor(ratio))
    return nf if abs(ratio - nf) < 1e-14 else n


def explicit_transport(A, bcv, cfl, c0, output_times, bc_switch=()):
    """Concentrations at output_times (increasing, from 0) of the explicit scheme
    c <- (I + dt A) c + dt bcv (ConvectionTransport::compute_one_step, transport.cc:593-716),
    with dt fixed over each interval between outputs (set_target_time + fix_dt_until_mark:
    interval / step_count).  bc_switch lists (time, boundary term) pairs in increasing time:
    the step that starts at t uses the term of the last pair with time <= t, and `bcv` before
    the first one -- the data are set to the last computed time before the step
    (transport.cc:600, 621-622) and the time advances after (:665)."""
    c = np.array(c0, np.float64)
    t = 0.0
    out = []

    def term(t0):
        cur = bcv
        for ts, v in bc_switch:
            if ts <= t0:
                cur = v
        return cur

    for target in output_times:
        if target > t:
            n = step_count(target - t, cfl)
            dt = (target - t) / n
            for i in range(n):
                c = c + dt * (A @ c) + dt * term(t + i * dt)
            t = target
        out.append(c.copy())
    return np.array(out)
