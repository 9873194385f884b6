"""The flow field text output (mh_raw_output_write, output_internal_flow_data of
darcy_flow_mh_output.cc:793-829) on CPU: written from the oracle's t01 solution and element flux
vectors, it has the reference's block layout and the reference's printed values (%.8g) for
every element of tests/01_steady_flow_123d."""
import numpy as np

import mhdarcy
import oracle as O
import topology as T
from helpers import fixture_bc, fixture_coeffs, load_fixture, oracle_problem

HEADER = ["// fields:",
          "//ele_id    ele_presure    flux_in_barycenter[3]    n_sides   side_pressures[n]    side_fluxes[n]"]


def t01_output(tmp_path, append_twice=False):
    z, mesh = load_fixture("t01")
    topo = T.build(mesh)
    P = oracle_problem(mesh, topo, topo["n_edges"], fixture_coeffs(z), fixture_bc(z, topo))
    sol = O.solve_mh_direct(P)
    flux = O.element_flux(P, sol)
    path = tmp_path / "raw_output.txt"
    args = (sol, flux, topo["el_side_start"], topo["side_edge"])
    mhdarcy.write_raw_output(path, *args, el_id=z["el_id"])  # steady: T=inf, as the reference
    if append_twice:
        mhdarcy.write_raw_output(path, *args, el_id=z["el_id"], time=1.5, append=True)
    return z, sol, flux, path.read_text().split("\n")


def test_t01_raw_output_block(tmp_path):
    z, sol, flux, lines = t01_output(tmp_path)
    n = len(z["el_id"])
    assert lines[:2] == HEADER
    assert lines[2] == "$FlowField" and lines[3] == "T=inf " and lines[4] == str(n)
    assert lines[5 + n] == "$EndFlowField" and lines[6 + n] == "" and len(lines) == 8 + n
    tol = lambda ref: 1e-8 + 5e-9 * np.abs(ref)
    for e, line in enumerate(lines[5:5 + n]):
        assert line.endswith(" ")
        tok = line.split()
        ns = z["ref_n_sides"][e]
        assert int(tok[0]) == z["ref_el_id"][e] and int(tok[5]) == ns and len(tok) == 6 + 2 * ns
        # every number is printed "%.8g"
        assert all(t == "%.8g" % float(t) for t in tok[1:5] + tok[6:])
        vals = np.array([float(t) for t in tok])
        assert abs(vals[1] - z["ref_pressure"][e]) <= tol(z["ref_pressure"][e])
        assert np.all(np.abs(vals[2:5] - z["ref_flux"][e]) <= tol(z["ref_flux"][e]))
        sp, sf = vals[6:6 + ns], vals[6 + ns:]
        assert np.all(np.abs(sp - z["ref_side_pressure"][e, :ns]) <= tol(z["ref_side_pressure"][e, :ns]))
        assert np.all(np.abs(sf - z["ref_side_flux"][e, :ns]) <= tol(z["ref_side_flux"][e, :ns]))
    # a line " n_sides " separates the vector from the side values, as in the reference
    assert " %d " % z["ref_n_sides"][0] in lines[5]


def test_raw_output_append(tmp_path):
    z, sol, flux, lines = t01_output(tmp_path, append_twice=True)
    n = len(z["el_id"])
    assert lines.count("$FlowField") == 2 and lines.count("$EndFlowField") == 2
    # the second block starts right after the first one's closing blank line
    assert lines[7 + n:9 + n] == HEADER and lines[9 + n] == "$FlowField" and lines[10 + n] == "T=1.5 "
    assert lines[5:5 + n] == lines[12 + n:12 + 2 * n]
