"""The C++ drop-ins of include/linsys_cuda.hh, compiled into a small C++ caller
(tests/cpp/linsys_driver.cpp) and run as a separate process on the reference's test 01:

  * LinSys_CUDA receives the second Schur complement element by element through
    mat_set_values, as the reference's SchurComplement fills a LinSys (ALLOCATE pass, then ADD
    pass; src/la/linsys.hh:129-156): the assembled CSR equals the oracle's summed matrix
    (CPU); finalize + solve on the GPU gives the direct solution of that system (gpu);
  * DarcyFlowMH_Steady_CUDA: its constructor's topology equals the library's (CPU);
    update_solution + get_solution_vector and the MH_DofHandler accessors reproduce the FP64
    direct solve and the reference's raw output of test 01 (gpu).
"""
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import mhdarcy
import oracle as O
from helpers import fixture_bc, fixture_coeffs, load_fixture, oracle_problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(mhdarcy.LIB_PATH)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("linsys_bin") / "linsys_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "linsys_driver.cpp"), "-o", exe, "-L", LIBDIR, "-lmhdarcy",
           "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run(driver, mode, d, solve):
    r = subprocess.run([driver, mode, str(d), str(int(solve))], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stderr)


def t01_problem():
    z, mesh = load_fixture("t01")
    with mhdarcy.MHSystem(mesh) as s:
        topo = s.topology()
        n_edges = s.n_edges
    coeffs = fixture_coeffs(z)
    bc = fixture_bc(z, topo)
    return z, mesh, topo, coeffs, bc, oracle_problem(mesh, topo, n_edges, coeffs, bc)


def write_blocks(d, P):
    blocks, rhs = O.schur2_element_blocks(P)
    with open(d / "blocks.bin", "wb") as f:
        for rows, vals in blocks:
            f.write(np.int32(len(rows)).tobytes())
            f.write(np.ascontiguousarray(rows, np.int32).tobytes())
            f.write(np.ascontiguousarray(vals, np.float64).tobytes())
    np.array([P.n_edges], np.int64).tofile(d / "n.bin")
    rhs.tofile(d / "rhs_in.bin")
    return rhs


def write_mesh_case(d, mesh, coeffs, bc):
    mesh.nodes.astype(np.float64).tofile(d / "nodes.bin")
    mesh.el_dim.astype(np.int32).tofile(d / "el_dim.bin")
    mesh.el_nodes.astype(np.int32).tofile(d / "el_nodes.bin")
    mesh.bc_dim.astype(np.int32).tofile(d / "bc_dim.bin")
    mesh.bc_nodes.astype(np.int32).tofile(d / "bc_nodes.bin")
    for k in ("conductivity", "anisotropy", "cross_section", "sigma", "water_source_density"):
        np.ascontiguousarray(coeffs[k], np.float64).tofile(d / (k + ".bin"))
    bc["bc_type"].astype(np.int32).tofile(d / "bc_type.bin")
    for k, f in (("pressure", "bc_pressure"), ("flux", "bc_flux"), ("robin_sigma", "bc_robin_sigma")):
        np.ascontiguousarray(bc[k], np.float64).tofile(d / (f + ".bin"))


def test_linsys_assembly_matches_oracle(driver, tmp_path):
    z, mesh, topo, coeffs, bc, P = t01_problem()
    rhs = write_blocks(tmp_path, P)
    run(driver, "linsys", tmp_path, False)
    S, r = O.schur2(P)
    rp = np.fromfile(tmp_path / "csr_row_ptr.bin", np.int32)
    col = np.fromfile(tmp_path / "csr_col.bin", np.int32)
    val = np.fromfile(tmp_path / "csr_val.bin", np.float64)
    G = sp.csr_matrix((val, col, rp), shape=S.shape)
    assert np.array_equal(rp, S.indptr) and np.array_equal(col, S.indices)
    assert abs(G - S).max() <= 1e-15 * abs(S).max()
    assert np.array_equal(np.fromfile(tmp_path / "rhs.bin", np.float64), rhs)


def test_darcy_constructor_topology(driver, tmp_path):
    z, mesh, topo, coeffs, bc, P = t01_problem()
    write_mesh_case(tmp_path, mesh, coeffs, bc)
    run(driver, "darcy", tmp_path, False)
    sizes = np.fromfile(tmp_path / "sizes.bin", np.int64)
    with mhdarcy.MHSystem(mesh) as s:
        zz = s.sizes
        assert list(sizes) == [zz.n_elements, zz.n_sides, zz.n_edges, zz.n_boundaries, zz.n_neighbours, zz.schur_nnz]
    for k in ("el_side_start", "side_edge", "bdr_bc_element"):
        assert np.array_equal(np.fromfile(tmp_path / (k + ".bin"), np.int32), topo[k]), k


def test_linsys_rejects_entries_outside_the_pattern(driver, tmp_path):
    """An ADD-pass entry that the ALLOCATE pass did not record is an error (reported, the
    driver exits with its code), not a silent write; one inside the pattern is accepted."""
    z, mesh, topo, coeffs, bc, P = t01_problem()
    write_blocks(tmp_path, P)
    S, _ = O.schur2(P)
    inside = int(S.indices[S.indptr[0] + 1])
    far = int(np.nonzero(S.getrow(0).toarray().ravel() == 0)[0][-1])
    rec = lambda r, c: np.array([r, c], np.int32).tobytes() + np.float64(1.0).tobytes()
    (tmp_path / "extra_add.bin").write_bytes(rec(0, inside))
    run(driver, "linsys", tmp_path, False)
    (tmp_path / "extra_add.bin").write_bytes(rec(0, inside) + rec(0, far))
    r = subprocess.run([driver, "linsys", str(tmp_path), "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 3 and "outside the allocated pattern" in r.stderr


@pytest.mark.gpu
def test_linsys_solve_on_gpu(gpu, driver, tmp_path):
    z, mesh, topo, coeffs, bc, P = t01_problem()
    write_blocks(tmp_path, P)
    run(driver, "linsys", tmp_path, True)
    info = np.fromfile(tmp_path / "solve_info.bin", np.float64)
    assert info[0] == 0 and info[2] <= 1e-12, info
    x = np.fromfile(tmp_path / "x.bin", np.float64)
    S, r = O.schur2(P)
    lam = spla.spsolve(S.tocsc(), r)
    assert np.abs(x - lam).max() <= 1e-9 * np.abs(lam).max()
    # the edge pressures of the reference's own run (raw output, %.8g)
    full = O.resolve(P, x)
    ns, ne = P.n_sides, P.n_el
    assert np.abs(full[ns:ns + ne] - z["ref_pressure"]).max() < 1e-8


@pytest.mark.gpu
def test_darcy_update_solution_on_gpu(gpu, driver, tmp_path):
    z, mesh, topo, coeffs, bc, P = t01_problem()
    write_mesh_case(tmp_path, mesh, coeffs, bc)
    run(driver, "darcy", tmp_path, True)
    sol = np.fromfile(tmp_path / "solution.bin", np.float64)
    ref = O.solve_mh_direct(P)
    assert len(sol) == len(ref)
    assert np.abs(sol - ref).max() <= 1e-8 * np.abs(ref).max()
    acc = np.fromfile(tmp_path / "accessors.bin", np.float64)
    k = 0
    for e in range(len(mesh.el_dim)):
        assert abs(acc[k] - z["ref_pressure"][e]) < 1e-8 + 5e-9 * abs(z["ref_pressure"][e])
        k += 1
        for i in range(mesh.el_dim[e] + 1):
            q, p = acc[k], acc[k + 1]
            k += 2
            assert abs(q - z["ref_side_flux"][e, i]) < 1e-8 + 5e-9 * abs(z["ref_side_flux"][e, i])
            assert abs(p - z["ref_side_pressure"][e, i]) < 1e-8 + 5e-9 * abs(z["ref_side_pressure"][e, i])
