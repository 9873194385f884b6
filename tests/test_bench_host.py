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


def test_bench_batch_case_shards():
    """bench.py's cfg3 batch over the instances a rank owns: one handle with one instance per
    id, the union mesh and the coefficients of every instance (host side, no GPU)."""
    bench = load_bench()
    from mhdarcy import parallel
    ids = parallel.shard(5, 1, 2)  # rank 1 of 2 owns instances 3 and 4
    system, mesh, coeffs = bench.batch_case(ids)
    with system:
        assert system.n_instances == len(ids) == 2
        assert len(coeffs["conductivity"]) == mesh.n_elements == system.n_elements


def test_bench_cpu_baseline_entry():
    """bench.py's cpu_baseline object (the CPU restatement on the workload, all threads and one
    thread) for Jacobi and ILU(3) CG, on cfg1 (complete solves fit the budget)."""
    bench = load_bench()
    cp = bench.CpuProblem(1)
    for pre in ("jacobi", "ilu3"):
        a = SimpleNamespace(config=1, cpu_precond=pre, cpu_budget_s=20.0)
        e = bench.cpu_baseline_entry(a, cp)
        assert e["value"] > 0 and e["cores"] >= 1 and e["kind"] == "port"
        assert e["one_core"]["cores"] == 1 and e["one_core"]["value"] > 0
        assert "complete solves" in e["sample"]


def test_bench_reference_arm_complete_and_projected(monkeypatch):
    """The reference arm on cfg1: complete solves when they fit the budget; when only one fits
    its cap, that one complete solve (steps 1, warm-up 0, the requested counts beside them); with
    no cap and a small budget, bounded samples projected with the recorded complete-solve
    iteration count.  Its config equals the GPU arm's for the same workload (sizes from the
    library)."""
    bench = load_bench()
    a = SimpleNamespace(config=1, cpu_precond="jacobi", steps=2, warmup=1, ref_budget_s=60.0, gpus=1,
                        ref_single_cap_s=400.0)
    out = bench.run_reference(a)
    assert out["impl"] == "reference" and out["value"] > 0 and out["projected"] is False
    assert out["e2e"]["value"] == out["value"] and out["cpu_baseline"]["kind"] == "port"
    assert out["ms_per_step"] > 0 and out["steps"] == 2 and out["warmup"] == 1
    from mhdarcy.cases import make_case
    mesh, _ = make_case(1)
    with mhdarcy.MHSystem(mesh) as s:
        z = s.sizes
        assert out["config"] == bench.workload_config(1, z.n_edges, z.schur_nnz, z.mh_size, z.n_elements)
    monkeypatch.setattr(bench, "cpu_full_record", lambda cfg, pre: {"iterations": 1630})
    a = SimpleNamespace(config=1, cpu_precond="jacobi", steps=2, warmup=1, ref_budget_s=0.05, gpus=1,
                        ref_single_cap_s=400.0)
    one = bench.run_reference(a)
    assert one["projected"] is False and one["steps"] == 1 and one["warmup"] == 0
    assert one["steps_requested"] == 2 and "one complete solve" in one["cpu_baseline"]["sample"]
    assert abs(one["value"] - 1e3 / one["ms_per_step"]) <= 1e-3 * one["value"]
    a = SimpleNamespace(config=1, cpu_precond="jacobi", steps=2, warmup=1, ref_budget_s=0.05, gpus=1,
                        ref_single_cap_s=0.0)
    out2 = bench.run_reference(a)
    assert out2["projected"] is True and "projected" in out2["cpu_baseline"]["sample"]
    # the projection of a 1630-iteration solve lands near the measured complete solve
    assert 0.2 < out2["value"] / out["value"] < 5.0


def test_bench_reference_arm_loads_no_product_library():
    """The reference arm builds and solves the workload with the oracle alone: the GPU
    library's shared object is never loaded into its process."""
    import subprocess
    import sys
    code = ("import sys, json; sys.path.insert(0, %r); import bench; from types import SimpleNamespace as N; "
            "o = bench.run_reference(N(config=1, cpu_precond='jacobi', steps=1, warmup=0, ref_budget_s=30.0, gpus=1, "
            "ref_single_cap_s=400.0)); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'v': o['value'], 'lib': 'libmhdarcy' in maps, 'orc': 'libmhoracle' in maps}))" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    import json
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["v"] > 0 and d["orc"] and not d["lib"]


def test_bench_setup_timing_isolated():
    """The child-process wrapper the bench line uses returns the same record."""
    r = load_bench().setup_timing_isolated(n=6, reps=1, timeout_s=600)
    assert "error" not in r, r
    assert r["elements"] == 6 * 6 ** 3 + 2 * 6 * 6 + 6
