#!/usr/bin/env python
"""Benchmark: steady MH Darcy solves/s to relative residual 1e-10 on one B200.

Workload (default, --config 5): the n=96 fractured Kuhn cube -- 5,308,416 tetrahedra, six
axis-aligned fracture planes at seeded grid positions (their triangles: cross-section 1e-3,
log10 K ~ U(-4,-2) per plane) and four 1D channels along grid lines inside fracture planes
(cross-section 1e-4, K = 1e-2); matrix log10 K ~ N(-7, 2) Gaussian-correlated with correlation
length 0.05, clipped to 1e-9..1e-2; Dirichlet p=1 at x=0 / p=0 at x=1.  10,950,146 edge
unknowns.  Synthetic and seeded: there is no public dataset for this path.  --config 1..4 select
the other workloads (2: the n=64 cube with one fracture and one channel).

A step is one full solve: local MH assembly + both Schur eliminations (K1), the Krylov solve
of the edge system to FP64 true relative residual <= 1e-10 (Jacobi-scaled and unscaled), and
back-substitution of element pressures and side fluxes (K4), with mesh, coefficients and
boundary data resident in HBM.  Methods (--methods): pcg64 (plain FP64 Jacobi-PCG, the
baseline), amg (aggregation-multigrid-preconditioned flexible CG, FP32/FP16 inner iteration,
FP64 residual replacements), fcg (the same with the learned smoother, trained first on a
smaller system of the same family), ir32, cheb.  `value` is the fastest converged method;
every method's row, its speed-up over pcg64 and its flux and pressure errors (at r_tol 1e-10
and 1e-12, against a solve to 1e-14) are in the line.  `e2e` times the fastest method through
the public API with host buffers: coefficients and boundary data copied in from pinned memory
every step and the full MH solution copied back.

--impl reference times the CPU path: the FP64 C restatement of the reference in oracle/ (OpenMP
over all host threads; Jacobi-preconditioned CG, or --cpu-precond ilu3 for the reference's own
ILU(3)), on the same workload built by the oracle alone (numpy mesh, C topology; no GPU
library).  Complete solves when they fit the time budget, else bounded samples projected with
the iteration count of a complete CPU solve recorded by oracle/cpu_full_solves.py.
Multi-GPU (torchrun): independent replicas, one per GPU, no data-path collective (--config 3:
one fixed batch sharded over the ranks).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "svn-export_b200"))

METRIC = "MH Darcy solves/s to 1e-10 residual: learned+FP32 vs plain FP64 PCG, 1 B200"
R_TOL = 1e-10
WORKLOADS = {
    1: "n=16 fractured Kuhn cube: 24,576 tets + 512 fracture triangles + 16 channel segments, log10 K ~ N(-6,1)",
    2: "n=64 fractured Kuhn cube: 1,572,864 tets + 8,192 fracture triangles + 64 channel segments, "
       "log10 K ~ N(-6,1.5) correlated (length 0.1)",
    3: "batch of uneven fractured cubes (n in {8,12,16,24,32}, one z=0.5 fracture each), log10 K ~ N(-6,1) "
       "correlated (length 0.05..0.2), all instances in one launch sequence",
    4: "n=48 fractured Kuhn cube: 663,552 tets + 4,608 fracture triangles, log10 K ~ N(-6,1)",
    5: "n=96 cube: 5,308,416 tets, 6 fracture planes, 4 channels, log10 K ~ N(-7,2) correlated (0.05)",
}
# solver ids of mh_darcy.h (MH_SOLVER_*) and per-method options
METHOD_IDS = {"pcg64": 0, "ir32": 1, "cheb": 2, "fcg": 3, "amg": 4}
SOLVE_KW = {"amg": lambda a: {"inner_rtol": a.amg_inner_rtol}, "fcg": lambda a: {"inner_rtol": a.amg_inner_rtol}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=5, choices=sorted(WORKLOADS))
    ap.add_argument("--methods", default="pcg64,amg,fcg",
                    help="comma list of pcg64, ir32, amg (multigrid FCG), cheb (Chebyshev-Jacobi FCG), "
                         "fcg (multigrid FCG with the learned smoother)")
    ap.add_argument("--amg-inner-rtol", type=float, default=1e-3,
                    help="FP32 residual reduction between FP64 replacements in the multigrid solves")
    ap.add_argument("--train-n", type=int, default=24, help="cube size of the system the network trains on")
    ap.add_argument("--train-epochs", type=int, default=30)
    ap.add_argument("--train-steps", type=int, default=20,
                    help="--unsteady: steps solved with the plain multigrid before the learned method trains")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the flux/pressure error block")
    ap.add_argument("--pcg-accuracy", action="store_true", help="also time pcg64 at r_tol 1e-12 in the error block")
    ap.add_argument("--extra-config", default="2,3",
                    help="comma list of further workloads timed with fewer steps, reported under `extra` (0: none)")
    ap.add_argument("--extra-unsteady", type=int, default=100, metavar="K",
                    help="also time the cfg4 unsteady protocol for K steps under extra.cfg4_unsteady (0: none)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-precond", choices=["jacobi", "ilu0", "ilu3"], default="jacobi",
                    help="preconditioner of the CPU path's CG: Jacobi (threaded throughout; the faster CPU solve on "
                         "multi-core hosts at the benchmark sizes) or ILU(k) (the reference's PETSc solver uses "
                         "ILU(3); sequential triangular solves)")
    ap.add_argument("--cpu-budget-s", type=float, default=20.0, help="CPU work of the cpu_baseline sample")
    ap.add_argument("--ref-budget-s", type=float, default=150.0,
                    help="CPU work of all warm-up and timed steps of --impl reference")
    ap.add_argument("--ref-single-cap-s", type=float, default=400.0,
                    help="--impl reference: when the steps of complete solves exceed the budget, time one complete "
                         "solve if it is estimated below this many seconds (0: project from a bounded sample instead)")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-setup-timing", action="store_true",
                    help="skip the host setup timing (gmsh read and handle creation at 56k elements)")
    ap.add_argument("--instances", type=int, default=256, help="batch size of --config 3 (over all ranks)")
    ap.add_argument("--accuracy", action="store_true",
                    help="flux and pressure errors of AMG and FP64 PCG solves at r_tol 1e-10 and 1e-12 against "
                         "an AMG solve driven to r_tol 1e-14 (full-size systems have no direct solve)")
    ap.add_argument("--unsteady", type=int, default=0, metavar="K",
                    help="time K implicit Euler steps (dt 0.01, time-varying boundary pressure) instead of "
                         "steady solves; reports steps/s")
    return ap.parse_args()


def load_json(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


# ---------------------------------------------------------------- clocks ----------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- roofline -----------------
AMG_DEGREE = 2  # Chebyshev smoothing degree of the AMG cycle (library default)
# the cycle reads the fine matrix's values in FP16 unless MH_AMG_HALF=0 (library default 1)
AMG_VALUE_BYTES = 4 if os.environ.get("MH_AMG_HALF", "1") == "0" else 2


def algorithmic_bytes(kernel, N, Z):
    """Bytes each launch must move at minimum (every array once; no padding, no re-reads).
    spmv:    values + column indices of the Z nonzeros, p (gathered, counted once), r read, q written.
    update:  x, r, p read and written, q read.
    smooth0: AMG Chebyshev step on the fine level (unit diagonal): values (FP16 copy, or FP32)
             + indices, x (or b) gathered, b read, x and d written; d read by the steps that
             continue a sequence (the fused first pre-smoothing pass and the first post-smoothing
             step start one): mean over the 2d-1 fine steps of one cycle."""
    if kernel == "smooth0":
        steps = 2 * AMG_DEGREE - 1
        reads_d = max(0, AMG_DEGREE - 2) + (AMG_DEGREE - 1)
        return Z * (4 + AMG_VALUE_BYTES) + 16 * N + 4 * N * reads_d / steps
    s = 8 if kernel.endswith("64") else 4
    if kernel.startswith("spmv"):
        return Z * (s + 4) + 3 * s * N
    return 7 * s * N


KERNEL_NAMES = {"spmv64": "k_cg_spmv<double>", "update64": "k_cg_update<double>", "spmv32": "k_cg_spmv<float>",
                "update32": "k_cg_update<float>", "smooth0": "k_sm_step (AMG fine level)"}


def roofline(stats_list, N, Z, peaks):
    """Roofline of the timed kernel class with the largest total device time (classes 0-4 of
    mh_solve_stats; class 5 is a whole V-cycle, reported beside it)."""
    names = ["spmv64", "update64", "spmv32", "update32", "smooth0"]
    nk = len(names)
    tot = [0.0] * 6
    cnt = [0] * 6
    for st in stats_list:
        for k in range(6):
            tot[k] += st["kernel_ms"][k]
            cnt[k] += st["kernel_count"][k]
    k = max(range(nk), key=lambda i: tot[i])
    if cnt[k] == 0:
        return None
    per_launch_s = tot[k] / cnt[k] / 1e3
    bytes_ = algorithmic_bytes(names[k], N, Z)
    achieved = bytes_ / per_launch_s / 1e9
    peak = peaks.get("hbm_gbs") if peaks else None
    peak_note = "measured"
    if not peak:
        peak, peak_note = 6650.0, "fallback"
    traffic = None
    tj = load_json(os.path.join(ROOT, "profiles", "traffic.json"))
    tkey = names[k] + ("_f16" if names[k] == "smooth0" and AMG_VALUE_BYTES == 2 else "")
    if tj and tkey in tj.get("bytes_per_unit", {}):
        traffic = tj["bytes_per_unit"][tkey] * (N if tj.get("unit") == "row" else 1)
    share = {names[i]: round(tot[i] / max(sum(tot[:nk]), 1e-30), 4) for i in range(nk) if cnt[i]}
    out = {"bound": "hbm", "kernel": KERNEL_NAMES[names[k]],
           "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
           "peak_source": peak_note, "traffic": traffic, "algorithmic_bytes_per_launch": int(bytes_),
           "avg_launch_us": round(per_launch_s * 1e6, 3), "launches": cnt[k], "time_share": share}
    if cnt[5]:
        out["vcycle_avg_us"] = round(tot[5] / cnt[5] * 1e3, 2)
        out["smooth0_share_of_vcycle"] = round(tot[4] / tot[5], 4) if tot[5] > 0 else None
    return out


# ---------------------------------------------------------------- unsteady --------------
def run_unsteady(a, rank, world):
    print(json.dumps(unsteady_line(a)), flush=True)


def unsteady_line(a):
    """K steps of the unsteady MH system (mh_unsteady_step: right-hand side from the previous
    pressures, solve, back-substitution) with the boundary pressure on x = 0 following
    1 + 0.5 sin(2 pi t); each method starts from zero pressure.  The matrix is the same in every
    step (same dt), so the multigrid hierarchy is built once and reused.  The learned method
    (fcg) runs the first --train-steps steps with the plain multigrid, trains the network on the
    system of the last of them (pairs from the plain solver) and solves the remaining steps with
    it; every method's steps after that point are timed as the window the comparison is made on."""
    import numpy as np
    import torch

    import mhdarcy
    from mhdarcy.cases import dirichlet_x_bc, make_case

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    stream = torch.cuda.Stream()
    mesh, coeffs = make_case(a.config)
    dt = 0.01
    k0 = min(a.train_steps, a.unsteady - 1)
    out = {}
    with mhdarcy.MHSystem(mesh) as s:
        s.set_stream(stream.cuda_stream)
        bc, left = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

        def rec(e):
            with torch.cuda.stream(stream):
                e.record(stream)

        for name in a.methods.split(","):
            kw = SOLVE_KW.get(name, lambda a: {})(a)

            def run(k, record=False):
                s.set_bc(bc["bc_type"], bc["pressure"])
                s.unsteady_init(dt, init_pressure=np.zeros(s.n_elements), lumped=False)
                p = bc["pressure"].copy()
                its, training = [], None
                if record:
                    rec(ev[0])
                for i in range(1, k + 1):
                    p[left] = 1.0 + 0.5 * np.sin(2 * np.pi * i * dt)
                    s.set_bc(bc["bc_type"], p)
                    m = METHOD_IDS[name]
                    if name == "fcg" and i <= k0:
                        m = METHOD_IDS["amg"]
                    st = s.unsteady_step(dt, method=m, r_tol=R_TOL, **kw)
                    if st["status"] not in (0, mhdarcy.MH_FELL_BACK):
                        raise RuntimeError(f"{name} step {i}: {st}")
                    its.append(st["iterations"])
                    if i == k0:
                        if record:
                            rec(ev[1])
                        if name == "fcg":
                            training = s.learned_train(n_pairs=12, epochs=a.train_epochs, lr=2e-3)
                        if record:
                            rec(ev[2])
                if record:
                    rec(ev[3])
                return its, training

            if name == "fcg":
                s.reset_learned()
            run(max(3, a.warmup))
            if name == "fcg":  # the timed run trains from the initial network again
                s.reset_learned()
            torch.cuda.synchronize()
            its, training = run(a.unsteady, record=True)
            torch.cuda.synchronize()
            ms_all = ev[0].elapsed_time(ev[3])
            ms_win = ev[2].elapsed_time(ev[3])
            nwin = a.unsteady - k0
            out[name] = {"steps_per_s": round(a.unsteady / (ms_all / 1e3), 3),
                         "window_steps": [k0 + 1, a.unsteady],
                         "window_steps_per_s": round(nwin / (ms_win / 1e3), 3),
                         "ms_per_step_window": round(ms_win / nwin, 3),
                         "iterations_mean_window": round(float(np.mean(its[k0:])), 2),
                         "iterations_mean": round(float(np.mean(its)), 2), "iterations_max": int(max(its)),
                         "ms_training": round(ev[1].elapsed_time(ev[2]), 2) if name == "fcg" else 0.0}
            if training:
                out[name]["training"] = training
    best = max(out, key=lambda m: out[m]["window_steps_per_s"])
    line = {"metric": "MH Darcy unsteady steps/s (implicit Euler, residual 1e-10)",
            "value": out[best]["window_steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": a.unsteady,
            "warmup": max(3, a.warmup), "ms_per_step": out[best]["ms_per_step_window"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": method_dtype(best, AMG_VALUE_BYTES == 2),
            "data": "synthetic: seeded fractured Kuhn cube, log-normal conductivity (no public dataset)",
            "config": {"workload": "cfg%d: %s, dt %g, %d steps" % (a.config, WORKLOADS[a.config], dt, a.unsteady),
                       "window": "steps %d-%d (the learned method trains after step %d)" % (k0 + 1, a.unsteady, k0)},
            "method": best, "methods": out}
    return line


# ---------------------------------------------------------------- accuracy --------------
def run_accuracy(a):
    """Side fluxes and element pressures of solves at r_tol 1e-10 and 1e-12 against a solve to
    r_tol 1e-14 (both FP64 residual norms), relative to the largest reference value."""
    import numpy as np
    import torch

    import mhdarcy
    from mhdarcy.cases import dirichlet_x_bc, make_case

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    mesh, coeffs = make_case(a.config)
    rows = []
    with mhdarcy.MHSystem(mesh) as s:
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        s.assemble()
        amg = {"method": mhdarcy.MH_SOLVER_AMG, "inner_rtol": a.amg_inner_rtol}
        st = s.solve(r_tol=1e-14, max_it=20000, **amg)
        ref = s.solution()
        ns, ne = s.n_sides, s.n_elements
        rows.append({"method": "amg", "r_tol": 1e-14, "status": st["status"], "iterations": st["iterations"],
                     "rel_residual": st["rel_residual"], "rel_residual_unscaled": st["rel_residual_unscaled"]})
        for name, kw in (("amg", amg), ("pcg64", {"method": mhdarcy.MH_SOLVER_PCG64})):
            for rt in (1e-10, 1e-12):
                st = s.solve(r_tol=rt, max_it=50000, **kw)
                sol = s.solution()
                rows.append({"method": name, "r_tol": rt, "status": st["status"], "iterations": st["iterations"],
                             "flux_err": float(np.abs(sol[:ns] - ref[:ns]).max() / np.abs(ref[:ns]).max()),
                             "pressure_err": float(np.abs(sol[ns:ns + ne] - ref[ns:ns + ne]).max()
                                                   / np.abs(ref[ns:ns + ne]).max())})
    print(json.dumps({"config": "cfg%d: %s" % (a.config, WORKLOADS[a.config]), "accuracy": rows}), flush=True)


# ---------------------------------------------------------------- post-processing -------
def element_flux_timing(system, stream, sz, mesh, reps=20):
    """The element-centre flux vectors of the last solution (mh_get_element_flux_device),
    timed with CUDA events on the handle's stream: mean of `reps` launches after one warm-up.
    Algorithmic bytes per launch: node coordinates once (24 per node), per element its node
    ids, side fluxes, side offset, cross-section and list entry read and 24 bytes written."""
    import ctypes as C

    import numpy as np
    import torch

    from mhdarcy import _lib
    ne = sz.n_elements
    buf = torch.empty((ne, 3), dtype=torch.float64, device="cuda")
    call = lambda: _lib.check(_lib.lib.mh_get_element_flux_device(system.h, C.c_void_p(buf.data_ptr()), buf.numel()),
                              system.h)
    call()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(reps):
        call()
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    nsides = np.asarray(mesh.el_dim) + 1
    algo = 24 * sz.n_nodes + int(np.sum(4 * nsides + 8 * nsides)) + ne * (4 + 8 + 4 + 24)
    ef = {"kernel": "k_element_flux (make_element_vector)", "ms_per_call": round(ms, 4),
          "algorithmic_bytes": algo, "achieved_gbs": round(algo / (ms / 1e3) / 1e9, 1),
          "note": "per call: element kernels plus one stream synchronisation"}
    # the transport's convection matrix (mh_transport_matrix_device): pattern built by the first
    # call, then values only; bytes per slot: kind, two side indices and the value (4+4+4+8),
    # per row its offset, sides, cross-section and the side fluxes read
    nnz = C.c_int64()
    _lib.check(_lib.lib.mh_transport_matrix(system.h, None, C.byref(nnz), None, None, None, None), system.h)
    tbuf = torch.empty(nnz.value, dtype=torch.float64, device="cuda")
    cfl = C.c_double()
    tcall = lambda: _lib.check(_lib.lib.mh_transport_matrix_device(system.h, None, C.c_void_p(tbuf.data_ptr()),
                                                                  nnz.value, C.byref(cfl)), system.h)
    tcall()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(reps):
        tcall()
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    tms = ev0.elapsed_time(ev1) / reps
    talgo = 20 * nnz.value + ne * (8 + 8) + 8 * int(np.sum(nsides)) + 8 * sz.n_edges
    tr = {"kernel": "k_transport_rows + k_edge_outflow (create_transport_matrix_mpi)", "nnz": nnz.value,
          "ms_per_call": round(tms, 4), "algorithmic_bytes": talgo,
          "achieved_gbs": round(talgo / (tms / 1e3) / 1e9, 1), "cfl_max_step": cfl.value,
          "note": "per call: two kernels, a 8-byte read-back and a stream synchronisation"}
    return {"element_flux": ef, "transport_matrix": tr}


# ---------------------------------------------------------------- host setup ------------
# Flow123d 1.7.0 on one process at 56,355 elements (bench_mel_table.tex:34,43,44), seconds
SETUP_PUBLISHED_S = {"GMSHReader - read mesh": 3.46, "MESH - setup topology": 0.49, "Darcy constructor": 3.28}


def setup_timing(n=21, reps=3):
    """Host-side setup at the size of the reference's published profile: a fractured n=21 cube
    (55,566 tets + 882 fracture triangles + 21 channel segments = 56,469 elements) written as a
    gmsh 2.2 file, read by the library's reader (mh_gmsh_read) and turned into a solver handle
    (MHSystem: topology, Schur pattern, SELL layout and device upload), each the median of
    `reps` host-timed runs."""
    import tempfile

    import numpy as np

    import mhdarcy
    mesh = mhdarcy.cube_mesh(n, [(2, n // 2)], [(0, n // 2, n // 2)])
    typ = np.array([15, 1, 2, 4])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "cube.msh")
        with open(path, "w") as f:
            f.write('$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n3\n3 3 "rock"\n2 2 "fracture"\n'
                    '1 1 "channel"\n$EndPhysicalNames\n$Nodes\n%d\n' % len(mesh.nodes))
            np.savetxt(f, np.column_stack([np.arange(1, len(mesh.nodes) + 1), mesh.nodes]),
                       fmt=["%d", "%.17g", "%.17g", "%.17g"])
            f.write("$EndNodes\n$Elements\n%d\n" % len(mesh.el_dim))
            dim = np.asarray(mesh.el_dim)
            for k in (3, 2, 1):  # cube_mesh orders tetrahedra, triangles, segments
                sel = np.where(dim == k)[0]
                cols = [sel + 1, typ[dim[sel]], np.full(len(sel), 2), np.full(len(sel), k), np.full(len(sel), k)]
                cols += [np.asarray(mesh.el_nodes)[sel, j] + 1 for j in range(k + 1)]
                np.savetxt(f, np.column_stack(cols), fmt="%d")
            f.write("$EndElements\n")
        size = os.path.getsize(path)
        t_read, t_create = [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            m = mhdarcy.read_gmsh(path)
            t_read.append(time.perf_counter() - t0)
        if not (np.array_equal(m.el_nodes, mesh.el_nodes) and np.array_equal(m.nodes, mesh.nodes)):
            raise RuntimeError("gmsh round trip changed the mesh")
    for _ in range(reps):
        t0 = time.perf_counter()
        s = mhdarcy.MHSystem(m)
        t_create.append(time.perf_counter() - t0)
        s.close()
    return {"elements": int(len(m.el_dim)), "gmsh_file_bytes": size, "host_threads": os.cpu_count(),
            "read_gmsh_s": round(statistics.median(t_read), 5), "create_s": round(statistics.median(t_create), 5),
            "reference_published_s": SETUP_PUBLISHED_S,
            "note": "host timers; read_gmsh = mh_gmsh_read + array copies, create = mh_create (topology, "
                    "Schur pattern, SELL layout, device upload); reference: Flow123d 1.7.0, 1 process, "
                    "56,355 elements"}


def setup_timing_isolated(n=21, reps=3, timeout_s=300):
    """setup_timing in a child process, so that nothing in it (a native fault included) can
    cost the bench line; an error is reported in place of the timings."""
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "print(json.dumps(bench.setup_timing(n=%d, reps=%d)))" % (ROOT, n, reps))
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout_s, cwd=ROOT)
        if r.returncode == 0:
            return json.loads(r.stdout.strip().splitlines()[-1])
        tail = (r.stderr.strip().splitlines() or [""])[-1]
        return {"error": "exit %d: %s" % (r.returncode, tail[:200])}
    except Exception as e:
        return {"error": "%s: %s" % (type(e).__name__, e)}


# ---------------------------------------------------------------- shared config ---------
def workload_config(cfg, n_edges, schur_nnz, mh_size, elements):
    """The `config` object of both benchmark arms: the workload and its sizes only (the
    method each arm runs is reported beside it)."""
    return {"workload": "cfg%d: %s" % (cfg, WORKLOADS[cfg]), "n_edges": int(n_edges), "schur_nnz": int(schur_nnz),
            "mh_size": int(mh_size), "elements": int(elements), "r_tol": R_TOL,
            "l2": "inputs larger than L2 (edge matrix %.0f MB in FP64 CSR)" % (schur_nnz * 12 / 1e6)}


def method_dtype(name, amg_half):
    """Arithmetic types a method computes in (FP64 true residual and updates in all)."""
    if name == "pcg64":
        return "f64"
    if name == "amg":
        return "f64+f32+f16" if amg_half else "f64+f32"
    if name == "fcg":
        return "f64+f32+f16+bf16" if amg_half else "f64+f32+bf16"
    return "f64+f32"


# ---------------------------------------------------------------- ours ------------------
def timed_solves(system, stream, method, k, warmup, kw, barrier, r_tol=R_TOL):
    """warmup untimed and k timed steps (assembly + solve + back-substitution) on the handle's
    stream; returns (ms per step on the device, stats of the last step, launches)."""
    import torch
    for _ in range(warmup):
        system.assemble()
        system.solve(method=method, r_tol=r_tol, **kw)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    l0 = system.kernel_launches()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(k):
        system.assemble()
        stats.append(system.solve(method=method, r_tol=r_tol, **kw))
    with torch.cuda.stream(stream):
        ev1.record(stream)
    barrier()
    return ev0.elapsed_time(ev1) / k, stats, system.kernel_launches() - l0


def batch_case(instance_ids):
    """The cfg3 batch of the given instances (each its own seeded uneven case) as one handle:
    (system, union mesh, concatenated coefficients)."""
    import numpy as np

    import mhdarcy
    from mhdarcy import parallel
    from mhdarcy.cases import make_case
    parts = [make_case(3, seed=parallel.case_seed(3, 0, i)) for i in instance_ids]
    system = mhdarcy.MHSystem.batch([m for m, _ in parts])
    coeffs = {k: np.concatenate([c[k] for _, c in parts]) for k in parts[0][1]}
    return system, system.mesh, coeffs


def run_extra_config(a, cfg, methods, barrier):
    """Another workload timed with fewer steps, reported under `extra` (cfg3: one step solves
    the whole batch of a.instances uneven instances)."""
    import numpy as np
    import torch

    import mhdarcy
    from mhdarcy import parallel
    from mhdarcy.cases import dirichlet_x_bc, make_case
    stream = torch.cuda.Stream()
    if cfg == 3:
        s, mesh, coeffs = batch_case(range(a.instances))
    else:
        mesh, coeffs = make_case(cfg)
        s = mhdarcy.MHSystem(mesh)
    out = {}
    with s:
        s.set_stream(stream.cuda_stream)
        bc, _ = dirichlet_x_bc(s.topology(), mesh)
        s.set_coeffs(**coeffs)
        s.set_bc(bc["bc_type"], bc["pressure"])
        sz = s.sizes
        per = s.n_instances
        for name in methods:
            kw = {"inner_rtol": a.amg_inner_rtol} if name == "amg" else {}
            ms, stats, _ = timed_solves(s, stream, METHOD_IDS[name], 5, 3, kw, barrier)
            out[name] = {"ms_per_step": round(ms, 3), "solves_per_s": round(per * 1e3 / ms, 3),
                         "iterations": stats[-1]["iterations"], "converged": stats[-1]["status"] in (0, 2)}
        cfg_d = workload_config(cfg, sz.n_edges, sz.schur_nnz, sz.mh_size, sz.n_elements)
        if cfg == 3:
            cfg_d["instances_per_step"] = per
        return {"config": cfg_d, "steps": 5, "warmup": 3, "methods": out}


def train_network(a, rank, system, cfg):
    """Trains the learned preconditioner once on a smaller system of the same family (the
    network depends on local matrix features only, so it transfers) and loads its weights
    into `system`."""
    import mhdarcy
    from mhdarcy.cases import dirichlet_x_bc, make_case
    tmesh, tcoeffs = make_case(cfg if cfg != 3 else 1, seed=4321 + rank, n=a.train_n)
    with mhdarcy.MHSystem(tmesh) as tsys:
        tbc, _ = dirichlet_x_bc(tsys.topology(), tmesh)
        tsys.set_coeffs(**tcoeffs)
        tsys.set_bc(tbc["bc_type"], tbc["pressure"])
        tsys.assemble()
        training = tsys.learned_train(n_pairs=12, epochs=a.train_epochs, lr=2e-3)
        training["train_edges"] = tsys.n_edges
        system.set_learned_weights(tsys.learned_weights())
    return training


def run_ours(a, rank, world):
    import numpy as np
    import torch

    import mhdarcy
    from mhdarcy import parallel
    from mhdarcy.cases import dirichlet_x_bc, make_case

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    # one process per GPU: independent replicas (or, for a batch, each rank's own share of the
    # instances); no collective on the data path, only the barrier and the max over ranks
    rank, world, dist = parallel.init("nccl", timeout_s=300) if world > 1 else (rank, world, None)
    stream = torch.cuda.Stream()
    if a.config == 3:
        # one fixed batch of a.instances uneven instances, sharded contiguously over the ranks
        system, mesh, coeffs = batch_case(parallel.shard(a.instances, rank, world))
    else:
        mesh, coeffs = make_case(a.config, seed=parallel.case_seed(a.config, rank))
        system = mhdarcy.MHSystem(mesh)
    per_step = system.n_instances
    system.set_stream(stream.cuda_stream)
    topo = system.topology()
    bc, _ = dirichlet_x_bc(topo, mesh)
    system.set_coeffs(**coeffs)
    system.set_bc(bc["bc_type"], bc["pressure"])
    sz = system.sizes
    N, Z = sz.n_edges, sz.schur_nnz
    system.assemble()
    tune = system.autotune(64) if not a.no_autotune else None

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return parallel.max_over_ranks(x, dist, device="cuda")

    names = [m for m in a.methods.split(",") if m]
    results = {}
    training = train_network(a, rank, system, a.config) if "fcg" in names else None
    clocks = ClockSampler(local) if not a.no_clocks else None
    for name in names:
        m = METHOD_IDS[name]
        kw = SOLVE_KW.get(name, lambda a: {})(a)
        if clocks and not results:
            barrier()
            clocks.start()
        ms, stats, launches = timed_solves(system, stream, m, a.steps, a.warmup, kw, barrier)
        ms = max_over_ranks(ms)
        ok = all(s["status"] in (0, mhdarcy.MH_FELL_BACK) for s in stats)
        # one more step with every Krylov kernel timed by in-graph CUDA events (for the
        # roofline; the events and per-graph read-backs add overhead, so not used for `value`)
        system.assemble()
        prof = [system.solve(method=m, r_tol=R_TOL, profile_kernels=True, **kw)]
        results[name] = {"ms_per_solve": ms, "solves_per_s": world * per_step / (ms / 1e3),
                         "iterations": stats[-1]["iterations"], "outer": stats[-1]["outer_iterations"],
                         "rel_residual": stats[-1]["rel_residual"],
                         "rel_residual_unscaled": stats[-1]["rel_residual_unscaled"], "converged": ok,
                         "ms_assembly": stats[-1]["ms_assembly"], "ms_backsub": stats[-1]["ms_backsub"],
                         "ms_precond_setup": stats[-1]["ms_setup"], "stats": prof, "launches": launches,
                         "dtype": method_dtype(name, AMG_VALUE_BYTES == 2), "fell_back": stats[-1]["fell_back"]}
        if name == "fcg":
            results[name]["training"] = training
        if name == "pcg64":
            # the whole Krylov solve against HBM: per iteration one FP64 SpMV (8 + 4 bytes per
            # slot, the row pointers, x read and q written) and 11 FP64 vector streams (p, x, r
            # updates and the Jacobi step), counted once each; assembly and back-substitution
            # left out (their own kernels, about 0.1% of the time)
            N, Z = sz.n_edges, sz.schur_nnz
            b_iter = Z * 12 + 4 * (N + 1) + 16 * N + 88 * N
            t_k = stats[-1]["ms_solve"] / 1e3
            gbs = stats[-1]["iterations"] * b_iter / t_k / 1e9
            pk = (load_json(os.path.join(ROOT, "MEASURED_PEAKS.json")) or {}).get("hbm_gbs") or 6650.0
            results[name]["hbm_per_solve"] = {
                "algorithmic_bytes_per_iteration": int(b_iter), "ms_krylov": round(1e3 * t_k, 3),
                "achieved_gbs": round(gbs, 1), "peak_gbs": pk, "frac": round(gbs / pk, 4)}
    clock_info = clocks.stop() if clocks else None
    best = max((r for r in results if results[r]["converged"]), key=lambda r: results[r]["solves_per_s"])
    rb = results[best]

    # accuracy: side fluxes and element pressures of every method's solve at r_tol 1e-10 and
    # 1e-12 against an AMG solve driven to 1e-14 (a full-size system has no direct solve); the
    # 1e-12 solve is timed too (the tolerance that meets a flux error of 1e-8 on these systems)
    accuracy = None
    if a.config != 3 and not a.no_accuracy:
        accuracy = {}
        st = system.solve(method=mhdarcy.MH_SOLVER_AMG, r_tol=1e-14, max_it=20000, inner_rtol=a.amg_inner_rtol)
        ref = system.solution()
        ns, ne = sz.n_sides, sz.n_elements
        accuracy["reference"] = {"method": "amg", "r_tol": 1e-14, "iterations": st["iterations"],
                                 "rel_residual": st["rel_residual"],
                                 "rel_residual_unscaled": st["rel_residual_unscaled"]}
        fmax, pmax = np.abs(ref[:ns]).max(), np.abs(ref[ns:ns + ne]).max()
        for name in names:
            kw = SOLVE_KW.get(name, lambda a: {})(a)
            for rt in (R_TOL, 1e-12):
                if rt != R_TOL and name == "pcg64" and not a.pcg_accuracy:
                    continue
                ms, stats, _ = timed_solves(system, stream, METHOD_IDS[name], 1, 0, kw, barrier, r_tol=rt)
                sol = system.solution()
                accuracy["%s@%g" % (name, rt)] = {
                    "ms_per_solve": round(ms, 3), "iterations": stats[-1]["iterations"],
                    "status": stats[-1]["status"],
                    "flux_err": float(np.abs(sol[:ns] - ref[:ns]).max() / fmax),
                    "pressure_err": float(np.abs(sol[ns:ns + ne] - ref[ns:ns + ne]).max() / pmax)}

    # end to end through the public API with host buffers
    ne = sz.n_elements
    pin = lambda arr, dt: torch.from_numpy(np.ascontiguousarray(arr, dtype=dt)).pin_memory().numpy()
    hc = {k: pin(v, np.float64) for k, v in coeffs.items()}
    hbt, hbp = pin(bc["bc_type"], np.int32), pin(bc["pressure"], np.float64)
    import ctypes as C

    from mhdarcy import _lib
    kwb = SOLVE_KW.get(best, lambda a: {})(a)
    # each step's solution goes to the host while the next step computes: a device-to-device
    # copy into one of two staging buffers (mh_get_solution_device), then a copy-engine transfer
    # into pinned host memory on a second stream; a staging buffer is reused only after its
    # transfer ended, and the timed region ends after the last transfer
    stage = [torch.empty(sz.mh_size, dtype=torch.float64, device="cuda") for _ in range(2)]
    hsol = [torch.empty(sz.mh_size, dtype=torch.float64).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    moved = [torch.cuda.Event(), torch.cuda.Event()]
    step_no = [0]

    def e2e_step():
        b = step_no[0] % 2
        step_no[0] += 1
        system.set_coeffs(**hc)
        system.set_bc(hbt, hbp)
        system.assemble()
        system.solve(method=METHOD_IDS[best], r_tol=R_TOL, **kwb)
        stream.wait_event(moved[b])
        _lib.check(_lib.lib.mh_get_solution_device(system.h, C.c_void_p(stage[b].data_ptr()), stage[b].numel()),
                   system.h)
        ready = torch.cuda.Event()
        ready.record(stream)
        copy_stream.wait_event(ready)
        with torch.cuda.stream(copy_stream):
            hsol[b].copy_(stage[b], non_blocking=True)
            moved[b].record(copy_stream)
    for _ in range(max(1, a.warmup - 1)):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(a.steps):
        e2e_step()
    stream.wait_stream(copy_stream)  # the last solution is on the host before the region ends
    with torch.cuda.stream(stream):
        ev1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(ev0.elapsed_time(ev1))
    # the host arrays copied in every step (absent fields are filled with defaults on the device)
    h2d = sum(v.nbytes for v in hc.values()) + hbt.nbytes + hbp.nbytes
    d2h = 8 * sz.mh_size
    peaks = load_json(os.path.join(ROOT, "MEASURED_PEAKS.json"))
    # Krylov kernels timed in-graph: the best method's, else the fastest timed one's
    timed = [r for r in results if any(st["kernel_count"][k] for st in results[r]["stats"] for k in range(5))]
    rstats = rb["stats"] if best in timed else (results[max(timed, key=lambda r: results[r]["solves_per_s"])]["stats"]
                                                 if timed else [])
    roof = roofline(rstats, N, Z, peaks) if rstats else None
    out = {
        "metric": METRIC, "value": round(rb["solves_per_s"], 4), "unit": "solves/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(rb["ms_per_solve"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": rb["dtype"],
        "data": "synthetic: seeded fractured Kuhn cube, log-normal conductivity (no public dataset)",
        "config": workload_config(a.config, N, Z, sz.mh_size, ne),
        "method": best, "instances_per_step": per_step,
        "method_note": ("value is the fastest converged method's (%s); every method's figure, the learned "
                        "one's (fcg) included, is under methods and speedup_vs_pcg64" % best),
        "parallelism": ("batch sharded over ranks" if a.config == 3 else "replicas") if world > 1 else "single GPU",
        "autotune": tune,
        "e2e": {"value": round(world * per_step * a.steps / (ms_e2e / 1e3), 4), "unit": "solves/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "inputs from pinned host memory through mh_set_coeffs / mh_set_bc every step; each "
                        "step's solution read back (mh_get_solution_device, then a pinned copy on a second "
                        "stream overlapping the next step); the region ends after the last read-back"},
        "roofline": roof,
        "gpu_launches": int(rb["launches"]),
        "methods": {k: {kk: vv for kk, vv in v.items() if kk != "stats"} for k, v in results.items()},
        "speedup_vs_pcg64": ({k: round(v["solves_per_s"] / results["pcg64"]["solves_per_s"], 3)
                              for k, v in results.items()} if "pcg64" in results else None),
        "accuracy": accuracy,
        "dofs_per_s": round(rb["solves_per_s"] / per_step * sz.mh_size, 1),
        "clocks": clock_info,
    }
    out["postprocess"] = element_flux_timing(system, stream, sz, mesh)
    system.close()
    extra = [int(c) for c in str(a.extra_config).split(",") if c.strip() not in ("", "0")]
    extra = [c for c in extra if c != a.config]
    if extra and world == 1:
        out["extra"] = {"cfg%d" % c: run_extra_config(a, c, ["pcg64", "amg"], barrier) for c in extra}
    if a.extra_unsteady > 0 and world == 1:
        # the unsteady protocol of cfg4 (train the learned method after step 20, compare steps
        # 21..K), as in --config 4 --unsteady K
        from types import SimpleNamespace
        u = SimpleNamespace(**vars(a))
        u.config, u.unsteady, u.warmup, u.methods = 4, a.extra_unsteady, 3, "pcg64,amg,fcg"
        out.setdefault("extra", {})["cfg4_unsteady"] = unsteady_line(u)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


# ------------------------------------------------------------ CPU path ------------------
def cpu_full_record(cfg, precond):
    """Iterations of a complete CPU solve of this configuration to r_tol 1e-10 with this
    preconditioner, measured by the CPU restatement itself (oracle/cpu_full_solves.py, which
    appends every run to oracle/cpu_full_solves.jsonl); None when not recorded."""
    rec = None
    try:
        with open(os.path.join(ROOT, "oracle", "cpu_full_solves.jsonl")) as f:
            for line in f:
                d = json.loads(line)
                if d.get("config") == cfg and d.get("precond") == precond and d.get("r_tol") == R_TOL \
                        and d.get("iterations", -1) > 0:
                    rec = d
    except OSError:
        pass
    return rec


class CpuProblem:
    """The workload built by the oracle alone (numpy mesh, C topology, C assembly): nothing of
    the GPU library is loaded.  The edge system's pattern is set-up work (not timed)."""

    def __init__(self, cfg):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np

        import cases as OC
        import oracle as O
        self.O = O
        self.cfg = cfg
        self.P, mesh, _, _, _ = OC.problem(cfg)
        S, _ = O.schur2(self.P)
        self.rp = np.ascontiguousarray(S.indptr, np.int32)
        self.col = np.ascontiguousarray(S.indices, np.int32)
        self.nnz = len(self.col)
        self.val = np.zeros(self.nnz)
        self.rhs = np.zeros(self.P.n_edges)
        del S

    def config(self):
        P = self.P
        return workload_config(self.cfg, P.n_edges, self.nnz, P.mh_size, P.n_el)

    def step(self, precond, iters):
        """One step: the threaded double-Schur assembly, `iters` iterations of preconditioned CG
        (None: to convergence at r_tol), and the back-substitution, each host-timed."""
        import scipy.sparse as sp
        O, P = self.O, self.P
        t0 = time.perf_counter()
        O.schur2_csr_into(P, self.rp, self.col, self.val, self.rhs)
        t_asm = time.perf_counter() - t0
        S = sp.csr_matrix((self.val, self.col, self.rp), shape=(P.n_edges, P.n_edges))
        rtol, max_it = (R_TOL, 200000) if iters is None else (1e-30, iters)
        t0 = time.perf_counter()
        t_factor = 0.0
        if precond == "jacobi":
            x, it, res = O.pcg_jacobi(S, self.rhs, rtol=rtol, max_it=max_it)
        else:
            x, it, res, t_factor, _ = O.pcg_iluk(S, self.rhs, k=int(precond[3:]), rtol=rtol, max_it=max_it)
        t_cg = time.perf_counter() - t0 - t_factor
        t0 = time.perf_counter()
        O.resolve(P, x)
        t_res = time.perf_counter() - t0
        done = max_it if iters is not None else it
        return {"t_asm": t_asm, "t_factor": t_factor, "t_iter": t_cg / max(1, done), "t_res": t_res,
                "iterations": done, "converged": iters is None and it > 0, "t_step": t_asm + t_factor + t_cg + t_res}


def cpu_runs(cp, precond, steps, warmup, budget_s, single_cap_s=0.0):
    """Times the CPU path: complete solves when (warmup + steps) of them fit the time budget;
    else, with single_cap_s, one complete solve (no warm-up) when it is estimated to fit that
    cap; else bounded samples (assembly, a number of CG iterations sized to the budget, and the
    back-substitution) whose per-iteration time is projected to the iteration count a
    complete CPU solve of this configuration needed (cpu_full_record).  Returns the measured
    steps and the solves/s, with how it was obtained."""
    probe = cp.step(precond, 10)
    rec = cpu_full_record(cp.cfg, precond)
    per_step = budget_s / max(1, steps + warmup)
    full_est = probe["t_asm"] + probe["t_res"] + probe["t_iter"] * (rec["iterations"] if rec else 1e9)
    complete = rec is None or full_est <= per_step
    if not complete and single_cap_s > 0 and full_est <= single_cap_s:
        run = cp.step(precond, None)
        t = run["t_step"]
        return {"value": 1.0 / t, "t_step_ms": t * 1e3, "complete": True,
                "how": "one complete solve to r_tol 1e-10 (%d iterations; %d steps would not fit the run, "
                       "estimated %.0f s each)" % (run["iterations"], steps + warmup, full_est),
                "runs": [run], "iterations_full": run["iterations"], "sample_iterations": None,
                "steps_timed": 1, "warmup_run": 0}
    if complete:
        iters = None
    else:
        iters = max(10, int((per_step - probe["t_asm"] - probe["t_res"]) / max(probe["t_iter"], 1e-9)))
        iters = min(iters, rec["iterations"])
    for _ in range(warmup):
        cp.step(precond, iters)
    runs = [cp.step(precond, iters) for _ in range(steps)]
    t_step = statistics.median(r["t_step"] for r in runs)
    if complete:
        value, how = 1.0 / t_step, "complete solves to r_tol 1e-10 (%d iterations)" % runs[-1]["iterations"]
        n_full = runs[-1]["iterations"]
    else:
        n_full = rec["iterations"]
        t_full = statistics.median(r["t_asm"] + r["t_res"] for r in runs) + \
            statistics.median(r["t_iter"] for r in runs) * n_full
        value = 1.0 / t_full
        how = ("projected: each step times the assembly, %d CG iterations and the back-substitution; the "
               "per-iteration time is multiplied by the %d iterations a complete CPU solve of this workload "
               "needed (oracle/cpu_full_solves.jsonl, measured by the CPU code itself)" % (iters, n_full))
    return {"value": value, "t_step_ms": t_step * 1e3, "complete": complete, "how": how, "runs": runs,
            "iterations_full": n_full, "sample_iterations": iters}


def cpu_baseline_entry(a, cp):
    """The `cpu_baseline` object of the bench line: the CPU path on all host threads (a bounded
    sample of about 20 s) and on one thread (per-iteration time from a short sample)."""
    O = cp.O
    r = cpu_runs(cp, a.cpu_precond, 1, 0, a.cpu_budget_s)
    cores = O.num_threads()
    O.set_threads(1)
    try:
        one = cp.step(a.cpu_precond, 10)
    finally:
        O.set_threads(cores)
    n_full = r["iterations_full"]
    one_value = 1.0 / (one["t_asm"] + one["t_res"] + one["t_iter"] * n_full) if n_full else None
    return {"value": round(r["value"], 6), "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": "cfg%d full mesh, %s-preconditioned CG (oracle/, OpenMP): %s" % (cp.cfg, a.cpu_precond, r["how"]),
            "one_core": {"value": round(one_value, 6) if one_value else None, "unit": "solves/s", "cores": 1,
                         "t_iter_s": one["t_iter"], "t_asm_s": one["t_asm"], "t_backsub_s": one["t_res"]},
            "detail": {k: r["runs"][-1][k] for k in ("t_asm", "t_factor", "t_iter", "t_res")}}


def run_reference(a):
    """The reference arm: the CPU restatement of the reference path (oracle/), all host
    threads, on this run's workload; rank 0 only (other ranks exit without work)."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return None
    cp = CpuProblem(a.config)
    r = cpu_runs(cp, a.cpu_precond, a.steps, a.warmup, a.ref_budget_s, a.ref_single_cap_s)
    v = round(r["value"], 6)
    cores = cp.O.num_threads()
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "solves/s", "n_gpus": a.gpus,
            "steps": r.get("steps_timed", a.steps), "warmup": r.get("warmup_run", a.warmup),
            "steps_requested": a.steps, "warmup_requested": a.warmup, "ms_per_step": round(r["t_step_ms"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded fractured Kuhn cube, log-normal conductivity (no public dataset)",
            "config": cp.config(), "method": "%s-pcg64 (CPU, oracle/)" % a.cpu_precond,
            "projected": not r["complete"],
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": r["how"]},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", a.gpus))
    if a.impl == "reference":
        out = run_reference(a)
        if out:
            print(json.dumps(out))
        return
    if a.accuracy:
        if rank == 0:
            run_accuracy(a)
        return
    if a.unsteady > 0:
        if rank == 0:
            run_unsteady(a, rank, world)
        return
    out = run_ours(a, rank, world)
    if rank == 0:
        if not a.no_cpu_baseline and world == 1 and a.config != 3:
            out["cpu_baseline"] = cpu_baseline_entry(a, CpuProblem(a.config))
        if world == 1 and not a.no_setup_timing:
            out["setup"] = setup_timing_isolated()
        print(json.dumps(out))


if __name__ == "__main__":
    main()
