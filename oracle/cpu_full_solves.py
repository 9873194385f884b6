"""TEST INFRASTRUCTURE ONLY: complete CPU solves of a benchmark configuration with the oracle
(no GPU library involved), timed on this host, printed as one JSON line per run and appended
to oracle/cpu_full_solves.jsonl.

A complete solve is what one benchmark step does: the element-local double-Schur assembly of
the edge system (threaded), preconditioned CG to relative residual r_tol on both FP64 norms
(Jacobi: threaded; ILU(k): threaded SpMV and updates, sequential triangular solves), and the
back-substitution (threaded).  The iteration counts it records are what bench.py's CPU arm
multiplies its per-iteration samples by when complete solves do not fit the benchmark run.

    python oracle/cpu_full_solves.py --config 2 --precond jacobi [--threads 8]
    python oracle/cpu_full_solves.py --config 5 --precond ilu3
"""
import argparse
import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


def full_solve(P, precond, r_tol):
    import numpy as np

    import oracle as O
    S, _ = O.schur2(P)                     # pattern (set-up, not timed)
    rp = np.ascontiguousarray(S.indptr, np.int32)
    col = np.ascontiguousarray(S.indices, np.int32)
    del S
    val = np.zeros(len(col))
    rhs = np.zeros(P.n_edges)
    t0 = time.perf_counter()
    O.schur2_csr_into(P, rp, col, val, rhs)
    t_asm = time.perf_counter() - t0
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, rp), shape=(P.n_edges, P.n_edges))
    t0 = time.perf_counter()
    t_factor, fill = 0.0, 1.0
    if precond == "jacobi":
        x, it, res = O.pcg_jacobi(A, rhs, rtol=r_tol, max_it=200000)
    else:
        x, it, res, t_factor, fill = O.pcg_iluk(A, rhs, k=int(precond[3:]), rtol=r_tol, max_it=200000)
    t_cg = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.resolve(P, x)
    t_res = time.perf_counter() - t0
    return {"iterations": it, "rel_residual": res, "t_assembly_s": t_asm, "t_factor_s": t_factor,
            "t_cg_s": t_cg - t_factor, "t_backsub_s": t_res, "t_solve_s": t_asm + t_cg + t_res, "fill": fill}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, required=True)
    ap.add_argument("--precond", default="jacobi", help="jacobi or iluK (e.g. ilu3)")
    ap.add_argument("--r-tol", type=float, default=1e-10)
    ap.add_argument("--threads", type=int, default=0, help="OpenMP threads (0: all)")
    ap.add_argument("--no-record", action="store_true")
    a = ap.parse_args()
    if a.threads:
        os.environ["OMP_NUM_THREADS"] = str(a.threads)
    import cases as OC
    import oracle as O
    P, mesh, coeffs, topo, bc = OC.problem(a.config)
    out = {"config": a.config, "precond": a.precond, "r_tol": a.r_tol, "n_edges": P.n_edges,
           "threads": O.num_threads(), "cpu": cpu_model(), "host_cpus": os.cpu_count()}
    out.update(full_solve(P, a.precond, a.r_tol))
    line = json.dumps(out)
    print(line, flush=True)
    if not a.no_record:
        with open(os.path.join(HERE, "cpu_full_solves.jsonl"), "a") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
