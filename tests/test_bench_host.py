"""bench.py's host-side pieces on CPU: the setup timing (gmsh write and read, handle creation)
and the cpu_baseline object for both CPU preconditioners, on small cubes (no GPU)."""
import importlib.util
import os
from types import SimpleNamespace

import mhdarcy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def test_bench_setup_timing():
    """bench.py's host setup timing (gmsh write, read, handle creation) runs on a small cube."""
    r = load_bench().setup_timing(n=6, reps=1)
    assert r["elements"] == 6 * 6 ** 3 + 2 * 6 * 6 + 6
    assert r["read_gmsh_s"] > 0 and r["create_s"] > 0 and r["gmsh_file_bytes"] > 0


def test_bench_cpu_baseline_entry():
    """bench.py's cpu_baseline object (the CPU restatement on the GPU run's workload) for both
    preconditioners, on a small cube."""
    bench = load_bench()
    from mhdarcy.cases import dirichlet_x_bc, make_case
    mesh, coeffs = make_case(1, n=6)
    with mhdarcy.MHSystem(mesh) as s:
        topo, n_edges = s.topology(), s.n_edges
    bc, _ = dirichlet_x_bc(topo, mesh)
    for pre, iters in (("jacobi", 50), ("ilu0", 10)):
        a = SimpleNamespace(config=1, cpu_sample_iters=5, cpu_precond=pre)
        e = bench.cpu_baseline_entry(a, (mesh, coeffs, bc, topo, n_edges), iters if pre == "jacobi" else None)
        assert e["value"] > 0 and e["detail"]["method"].startswith(pre)
        assert e["detail"]["iters"] == (iters if pre == "jacobi" else bench.ILU0_PCG_ITERS[1])


def test_bench_setup_timing_isolated():
    """The child-process wrapper the bench line uses returns the same record."""
    r = load_bench().setup_timing_isolated(n=6, reps=1, timeout_s=600)
    assert "error" not in r, r
    assert r["elements"] == 6 * 6 ** 3 + 2 * 6 * 6 + 6
