#!/usr/bin/env python
"""Headline benchmark: solves/s of the 3D variable-coefficient Poisson solve
-div(k grad u) = F on [0,1]^3 with 257^3 nodes, k log-normal (sigma=1) smoothed
by 3 box passes, F ~ N(0,1), mixed Dirichlet/Neumann/Robin(1,1,0) faces,
geometric-MG V(2,2)-preconditioned CG with red-black Gauss-Seidel, FP64, to
1e-10 relative residual (the reference's CPU path cannot express this
divergence-form problem; the CPU baseline is the oracle port of the same
algorithm).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

A step is one complete solve. `value` is measured with k and f resident in
HBM (device pointers); `e2e` goes through the same C-ABI call with pinned host
buffers, so every step includes the H2D copy of k and f and the D2H copy of the
solution. Multi-GPU runs are independent replicas (no collective on the data
path); each rank solves its own copy and the time is the max over ranks.

CPU sides: `cpu_baseline` is two whole converged solves of the same input by
the oracle port (oracle/restate.c) on all host cores; `--impl reference` times
W + K whole converged solves the same way; `forms.reference_code` times the
reference's own CPU code (oracle/_ref) where it has the method (2D CG and
Jacobi at 129^2, 2D projection at 256^2) beside the GPU. `summary`, last in
the line, repeats the forms' headline figures.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "solves/s (3D var-k Poisson 257^3, MG-PCG FP64 to 1e-10 rel. residual)"
UNIT = "solves/s"
N_DEFAULT = 257
SEED = 1234


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and serving measurements")
    return ap.parse_args()


def config(n, l2_note):
    return {"workload": f"3D variable-k Poisson {n}^3, MG V(2,2)-PCG red-black GS, FP64, rel. residual 1e-10",
            "grid": [n, n, n], "dofs": n ** 3, "k": "log-normal sigma=1, 3 box passes", "f": "N(0,1)",
            "faces": "left/right D0, bottom/top N0, front Robin(1,1,0), back D0", "seed": SEED,
            "parallelism": "replicas", "l2": l2_note}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_name):
    """DRAM bytes per launch of `kernel_name` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel_name:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region,
    every 200 ms: a query now and then holds the GPU's work up by tens of ms
    (measured on the 257^3 solve: about one run in four at 100 ms), so the
    sampling is no denser than the clocks record needs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation and the first query) is
        # its heaviest part: wait for the first sample before the caller's
        # timed region begins (at most 5 s)
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.01)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower().startswith("active")})
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ CPU side

def cpu_solve_times(prob, count):
    """Wall times of `count` whole converged solves of `prob` by the oracle port
    of the same MG-PCG (oracle/restate.c) on all host cores."""
    from oracle import oracle
    from pde_solver_b200 import abi
    from pde_solver_b200.problem import default_options

    cores = os.cpu_count() or 1
    oracle.build(ref=False)
    oracle.restate().rs_set_threads(cores)
    o = default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=400)
    times, iters = [], None
    for _ in range(count):
        t0 = time.perf_counter()
        st, _, rep = oracle.rs_solve(prob, o)
        times.append(time.perf_counter() - t0)
        if st != abi.OK:
            raise RuntimeError(f"oracle solve failed: {st}")
        iters = rep.iterations
    return times, iters, cores


def cpu_sample(prob, count=2):
    """CPU baseline beside the GPU line: `count` whole converged solves of the
    same input by the oracle port (the reference's CPU path has no 3D
    divergence-form MG-PCG), median wall time."""
    times, iters, cores = cpu_solve_times(prob, count)
    t = statistics.median(times)
    return {"value": 1.0 / t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"oracle/restate.c MG-PCG on the same {prob.nx}^3 input, OpenMP {cores} threads: "
                       f"{count} whole converged solves ({iters} iterations each), median "
                       f"{t:.2f}s (all: {', '.join(f'{v:.2f}' for v in times)} s)")}


def reference_code_paths(lib, abi, device):
    """Configurations where the reference's own CPU code exists, timed beside
    the GPU: 2D Poisson 129^2 with the MMS right side by CG (CgSolve) and by
    Jacobi (SolveJacobi2D) to the reference's own stopping rules, and the 2D
    pressure projection of a 256^2 N(0,1) velocity field (ProjectVelocity2D,
    CG to 1e-10 relative). CPU: oracle/_ref (the reference compiled from its
    sources), one whole call each, all host cores. GPU: the same call through
    the C ABI with host buffers (copies included), median of 5 after one warm-up."""
    from oracle import oracle
    from pde_solver_b200 import solver, synthetic
    from pde_solver_b200.problem import default_options

    if not oracle.have_reference():
        return {"unavailable": "oracle/_ref/libpderef.so not built"}
    cores = os.cpu_count() or 1
    oracle.reference().pderef_set_threads(cores)
    out = {"cores": cores, "kind": "reference"}
    for name, method, max_iter, tol in (("config1_cg_129", abi.CG, 8000, 1e-10),
                                        ("config1_jacobi_129", abi.JACOBI, 200000, 1e-10)):
        p = synthetic.poisson_mms_2d(129)
        p.f = None
        opt = default_options(method=method, max_iter=max_iter, tol=tol, device=device.index or 0)
        t0 = time.perf_counter()
        st, ref, _, err = oracle.ref_solve(p, opt, rhs_latex=synthetic.MMS_RHS_LATEX)
        cpu_s = time.perf_counter() - t0
        p.f = oracle.ref_materialize(synthetic.MMS_RHS_LATEX, p)
        got, rep = solver.solve(p, opt)
        ts = []
        for _ in range(5):
            torch_sync()
            t0 = time.perf_counter()
            got, rep = solver.solve(p, opt)
            ts.append(time.perf_counter() - t0)
        gpu_s = statistics.median(ts)
        d = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        out[name] = {"cpu_ms": 1e3 * cpu_s, "gpu_e2e_ms": 1e3 * gpu_s, "gpu_device_ms": rep.device_ms,
                     "speedup_e2e": cpu_s / gpu_s, "iterations": rep.iterations, "rel_l2_vs_reference": d,
                     "cpu_status": st}
    n = 256
    u, v, p0 = synthetic.projection_fields(n, seed=17)
    h = 1.0 / (n - 1)
    t0 = time.perf_counter()
    st, ur, vr, _, pr, rrep = oracle.ref_project(u, v, None, p0, n, n, 1, h, h, 1.0, 0.01, 20000, 1e-10)
    cpu_s = time.perf_counter() - t0
    solver.project_velocity(u, v, None, p0, n, n, 1, h, h, 1.0, 0.01, 20000, 1e-10)
    ts = []
    for _ in range(5):
        torch_sync()
        t0 = time.perf_counter()
        ug, vg, _, pg, rep = solver.project_velocity(u, v, None, p0, n, n, 1, h, h, 1.0, 0.01, 20000, 1e-10)
        ts.append(time.perf_counter() - t0)
    gpu_s = statistics.median(ts)
    out["projection_256"] = {"cpu_ms": 1e3 * cpu_s, "gpu_e2e_ms": 1e3 * gpu_s, "gpu_device_ms": rep.device_ms,
                             "speedup_e2e": cpu_s / gpu_s, "poisson_iterations": rep.poisson_iterations,
                             "cpu_poisson_iterations": int(rrep[0]),
                             "rel_l2_vs_reference": float(np.linalg.norm(pg - pr) / np.linalg.norm(pr))}
    return out


def torch_sync():
    import torch

    torch.cuda.synchronize()


TUNE_CACHE = os.path.join(ROOT, "pde_solver_b200", "batch_tune_cache.txt")


def bench_batched(lib, abi, n2d=2048, n3d=256, reps=3):
    """Batched form: 2048 2D grids (sides log-uniform in [33, 513]) and 256 3D
    grids (sides log-uniform in [17, 129]), k log-normal sigma=0.5, f ~ N(0,1),
    Dirichlet 0; FP32 MG-PCG in FP64 refinement to 1e-10 for every member; the
    schedule comes from the autotuner's cache. Compared with the plain FP64
    MG-PCG path (one pdeb200_solve per grid) on an evenly spaced sample."""
    import torch

    from pde_solver_b200 import synthetic
    from pde_solver_b200.batch import Batch
    from pde_solver_b200.problem import default_options

    ms = synthetic.batch_members(n2d, n3d)
    t0 = time.perf_counter()
    b = Batch(ms, autotune=1, tune_cache=TUNE_CACHE)
    create_s = time.perf_counter() - t0
    b.solve(1e-10)
    dev = []
    for _ in range(reps):
        reps_ = b.solve(1e-10)
        dev.append(b.stats.device_ms)
    st = b.stats
    worst = max(r.rel_residual for r in reps_)
    o = b.options()
    # end to end: packed f from pinned host memory in, packed solution out
    nodes = b.nodes
    f_host = torch.from_numpy(np.concatenate([p.f for p in ms])).pin_memory()
    x_host = torch.empty(nodes, dtype=torch.float64).pin_memory()
    t0 = time.perf_counter()
    for _ in range(reps):
        lib.pdeb200_batch_load_rhs(b.handle, C.c_void_p(f_host.data_ptr()), abi.MEM_HOST)
        b.solve(1e-10)
        lib.pdeb200_batch_read(b.handle, C.c_void_p(x_host.data_ptr()), abi.MEM_HOST)
    e2e_s = (time.perf_counter() - t0) / reps
    b.close()
    # plain FP64 path on every 36th member
    opt = default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=400)
    from pde_solver_b200 import solver

    sample = ms[::36]
    solver.solve(sample[0], opt)
    plain_ms = 0.0
    for p in sample:
        _, r = solver.solve(p, opt)
        plain_ms += r.device_ms
    plain_rate = len(sample) / (plain_ms / 1e3)
    batched_rate = len(ms) / (statistics.median(dev) / 1e3)
    return {"workload": f"{n2d} 2D grids (sides 33..513) + {n3d} 3D grids (sides 17..129), var-k Poisson",
            "members": len(ms), "nodes": nodes, "precision": "FP32 MG-PCG in FP64 refinement, tol 1e-10",
            "solves_per_s": batched_rate, "ms_per_batch": statistics.median(dev),
            "e2e_solves_per_s": len(ms) / e2e_s, "e2e_h2d_bytes": nodes * 8, "e2e_d2h_bytes": nodes * 8,
            "worst_rel_residual": worst, "converged": st.converged, "cycles": st.cycles,
            "kernel_launches": st.kernel_launches, "device_gb": st.device_bytes / 1e9, "create_s": create_s,
            "schedule": {"tile": [o.tile_x, o.tile_y, o.tile_z], "pre": o.pre_smooth, "post": o.post_smooth,
                         "inner_tol": o.inner_tol, "from_cache": bool(st.tuned_from_cache)},
            "plain_fp64_solves_per_s": plain_rate, "plain_fp64_sample": len(sample),
            "speedup_vs_plain_fp64": batched_rate / plain_rate}


def bench_output(field, n, reps=3):
    """Output and input forms around the solve, on the headline grid: the
    legacy ASCII VTK and the VTI (with the CLI's derived fields) files of the
    solution, formatted on the GPU and written to a tmpfs file (so the file
    system does not bound the number), and a LaTeX right side evaluated at
    every node on the GPU. The reference's CPU writers and per-node evaluator
    are timed on a 16-plane sample and scaled to the grid."""
    import tempfile

    import torch

    from pde_solver_b200 import solver
    from pde_solver_b200.problem import GridProblem

    p = GridProblem(n, n, n, bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), a=-1.0, b=-1.0, az=-1.0)
    tmp = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    out = {"grid": f"{n}^3", "file_system": "tmpfs" if tmp.startswith("/dev/shm") else "default temp dir"}
    try:
        for kind, fn in (("vtk_legacy", solver.write_vtk), ("vti_derived", solver.write_vti)):
            path = os.path.join(tmp, "out." + kind)
            fn(path, p, field.data_ptr())
            ts = []
            for _ in range(reps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                fn(path, p, field.data_ptr())
                ts.append(time.perf_counter() - t0)
            size = os.path.getsize(path)
            out[kind] = {"ms": 1e3 * statistics.median(ts), "mb": size / 1e6,
                         "file_gbs": size / statistics.median(ts) / 1e9}
            os.remove(path)
        latex = r"-3\pi^2\sin(\pi*x)\sin(\pi*y)\sin(\pi*z) + \exp(-(x^2+y^2+z^2))"
        dev = torch.empty(p.n, dtype=torch.float64, device=field.device)
        solver.eval_expression(latex, p, out=dev.data_ptr())
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            solver.eval_expression(latex, p, out=dev.data_ptr())
            ts.append(time.perf_counter() - t0)
        out["expression"] = {"latex": latex, "ms": 1e3 * statistics.median(ts),
                             "nodes_per_s": p.n / statistics.median(ts)}
        if oracle_available():
            from oracle import oracle

            ps = GridProblem(n, n, 16, bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), a=-1.0, b=-1.0, az=-1.0)
            fs = field[: ps.n].cpu().numpy()
            scale = n / 16.0
            t0 = time.perf_counter()
            oracle.ref_write_vtk(os.path.join(tmp, "r.vtk"), ps, fs)
            out["vtk_legacy"]["reference_cpu_ms"] = 1e3 * (time.perf_counter() - t0) * scale
            t0 = time.perf_counter()
            oracle.ref_write_vti(os.path.join(tmp, "r.vti"), ps, fs)
            out["vti_derived"]["reference_cpu_ms"] = 1e3 * (time.perf_counter() - t0) * scale
            t0 = time.perf_counter()
            oracle.ref_materialize(latex, ps)
            out["expression"]["reference_cpu_ms"] = 1e3 * (time.perf_counter() - t0) * scale
            out["reference_sample"] = (f"reference writers / ExpressionEvaluator (oracle/_ref) on {n}x{n}x16, "
                                       f"one host thread, scaled by {scale:.2f}")
            for k in ("vtk_legacy", "vti_derived", "expression"):
                out[k]["speedup_vs_reference_cpu"] = out[k]["reference_cpu_ms"] / out[k]["ms"]
    finally:
        for f in os.listdir(tmp):
            os.remove(os.path.join(tmp, f))
        os.rmdir(tmp)
    return out


def oracle_available():
    try:
        from oracle import oracle

        return oracle.have_reference()
    except Exception:
        return False


def bench_serving(abi, count=256, seed=7):
    """Serving form: a stream of Poisson requests (2D sides 65..513, 3D sides
    65..129, k log-normal sigma=0.5) submitted at once (saturation) to a
    server, mixed precision (continuous batching, 6 lanes) vs the plain FP64
    path (16 lanes); latency is submit -> result written to host memory."""
    from pde_solver_b200 import synthetic
    from pde_solver_b200.server import Server

    import copy

    import torch

    reqs = [s for s in synthetic.serving_requests(count, seed=seed, rate_hz=1e9, mix=(1.0, 0.0, 0.0))]
    probs = [synthetic.poisson_request_problem(sp["n"], sp["dim"], sp["seed"]) for _, _, sp in reqs]
    # device-resident state: k and f already in HBM (as a preceding device
    # stage would leave them), results written to device buffers
    dev = torch.device("cuda", 0)
    keep, dprobs, outs = [], [], []
    for p in probs:
        k = torch.from_numpy(p.k).to(dev)
        f = torch.from_numpy(p.f).to(dev)
        o = torch.empty(p.n, dtype=torch.float64, device=dev)
        q = copy.copy(p)
        q.k, q.f, q.mem_space, q.k_dev, q.f_dev = None, None, abi.MEM_DEVICE, k.data_ptr(), f.data_ptr()
        keep += [k, f]
        dprobs.append(q)
        outs.append(o)
    torch.cuda.synchronize()
    out = {}
    for mode, plist in (("device_resident", dprobs), ("host_inputs", probs)):
        res_mode = {}
        # each precision at its best lane setting on this box (swept): mixed
        # groups of at most 64 requests on 6 lanes, plain FP64 one request per
        # lane on 16; mixed_adaptive solves a request single-grid while fewer
        # than 8 wait
        for name, prec, lanes, single in (("mixed", abi.MIXED, 6, 0), ("mixed_adaptive", abi.MIXED, 6, 8),
                                          ("fp64", abi.FP64, 16, 0)):
            with Server(lanes=lanes, max_batch=64, precision=prec, single_below=single, tile_x=64, tile_y=64,
                        tile_z=32, pre_smooth=1, post_smooth=2, inner_tol=1e-5) as s:
                dv = mode == "device_resident"
                s.wait(s.submit_poisson(plist[0], out=outs[0].data_ptr() if dv else None))
                s.stats(reset=True)
                t0 = time.perf_counter()
                ids = [s.submit_poisson(p, out=outs[q].data_ptr() if dv else None) for q, p in enumerate(plist)]
                res = [s.wait(i)[1] for i in ids]
                wall = time.perf_counter() - t0
                st = s.stats()
            res_mode[name] = {"solves_per_s": len(plist) / wall, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                              "lanes": lanes,
                              "failed": int(sum(r.status != abi.OK for r in res)),
                              "max_group": int(max(r.group_size for r in res)),
                              "single_grid": int(sum(r.group_size == 1 for r in res))}
        res_mode["speedup_mixed_vs_fp64"] = res_mode["mixed"]["solves_per_s"] / res_mode["fp64"]["solves_per_s"]
        res_mode["speedup_mixed_adaptive_vs_fp64"] = (res_mode["mixed_adaptive"]["solves_per_s"] /
                                                      res_mode["fp64"]["solves_per_s"])
        out[mode] = res_mode
    out["workload"] = f"{count} Poisson requests at saturation (2D 65..513, 3D 65..129), tol 1e-10"
    return out


def bench_convdiff(lib, abi, device, n=513, seed=99, reps=2):
    """Convection-diffusion form: -eps Laplace(u) + b.grad(u) = F on n^3 nodes
    (eps 1e-2, b a seeded unit vector, F ~ U[-1,1], Dirichlet 0, centred
    convection), MG-preconditioned BiCGStab to 1e-10 relative residual in
    FP32 inside FP64 iterative refinement, beside the same solve in plain
    FP64; F resident in HBM. At 513^3 the mixed result's error is measured
    against the FP64 GPU solution; `vs_fp64_oracle` measures both GPU results
    against the FP64 oracle on the same workload at 129^3. The coefficients
    are constants, so there is no coefficient array for BF16 storage."""
    import copy

    import torch

    from pde_solver_b200 import synthetic
    from pde_solver_b200.problem import default_options

    p = synthetic.convection_diffusion_3d(n, seed)
    f_dev = torch.from_numpy(p.f).to(device)
    dp = copy.copy(p)
    dp.f, dp.mem_space, dp.f_dev = None, abi.MEM_DEVICE, f_dev.data_ptr()
    cp = dp.to_c()
    out, sols = {}, {}
    for name, prec in (("fp64", abi.FP64), ("mixed", abi.MIXED)):
        o = default_options(method=abi.MG_BICGSTAB, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=200,
                            device=device.index or 0, precision=prec)
        x = torch.empty(p.n, dtype=torch.float64, device=device)
        times = []
        for r in range(reps + 1):  # the first solve is warm-up
            rep = abi.Report()
            st = lib.pdeb200_solve(C.byref(cp), C.byref(o), C.c_void_p(x.data_ptr()), C.byref(rep))
            if st != abi.OK:
                raise RuntimeError(f"convection-diffusion {name} solve failed: {st} {rep.message.decode()}")
            if r:
                times.append(rep.device_ms)
        ms = statistics.median(times)
        sols[name] = x
        out[name] = {"solves_per_s": 1e3 / ms, "ms": ms, "iterations": rep.iterations,
                     "outer_iterations": rep.outer_iterations, "rel_residual": rep.rel_residual,
                     "dof_iterations_per_s": p.n * rep.iterations / (ms / 1e3), "launches": rep.kernel_launches}
    d = sols["mixed"] - sols["fp64"]
    out["mixed"]["rel_l2_vs_fp64"] = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(sols["fp64"]))
    out["mixed"]["max_abs_vs_fp64"] = float(d.abs().max())
    out["speedup_mixed_vs_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    out["workload"] = (f"3D convection-diffusion {n}^3, eps 1e-2, MG-BiCGStab to 1e-10 rel. residual, "
                       f"FP32-in-FP64 refinement vs FP64, F resident in HBM, median of {reps} solves")
    del sols, d, x, f_dev
    torch.cuda.empty_cache()
    try:
        out["vs_fp64_oracle"] = convdiff_oracle_check(abi)
    except Exception as exc:
        out["vs_fp64_oracle"] = {"error": str(exc)}
    return out


def convdiff_oracle_check(abi, n=129, seed=99):
    """Error of the GPU results of the convection-diffusion workload against
    the FP64 oracle at a size the host solves in seconds: the oracle port's
    unpreconditioned FP64 BiCGStab (oracle/restate.c, all host cores) to 1e-13
    relative residual on the same 129^3 system."""
    from oracle import oracle
    from pde_solver_b200 import solver, synthetic
    from pde_solver_b200.problem import default_options

    p = synthetic.convection_diffusion_3d(n, seed)
    oracle.build(ref=False)
    oracle.restate().rs_set_threads(os.cpu_count() or 1)
    bnorm = float(np.linalg.norm(p.f.reshape(n, n, n)[1:-1, 1:-1, 1:-1]))
    t0 = time.perf_counter()
    st, ref, rrep = oracle.rs_solve(p, default_options(method=abi.BICGSTAB, tol=1e-13 * bnorm, max_iter=20000))
    cpu_s = time.perf_counter() - t0
    if st != abi.OK:
        raise RuntimeError(f"oracle BiCGStab failed: {st}")
    res = {"grid": f"{n}^3", "oracle": "oracle/restate.c BiCGStab FP64 to 1e-13 rel.", "oracle_iterations":
           rrep.iterations, "oracle_s": cpu_s}
    for name, prec, bf16 in (("fp64", abi.FP64, 0), ("mixed", abi.MIXED, 0), ("mixed_bf16", abi.MIXED, 1)):
        got, rep = solver.solve(p, default_options(method=abi.MG_BICGSTAB, tol=1e-10, tol_mode=abi.TOL_RELATIVE,
                                                   max_iter=200, precision=prec, bf16_coefficients=bf16))
        res[name] = {"rel_l2_vs_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                     "rel_residual": rep.rel_residual}
    return res


def summarize(line):
    """Compact headline figures of every form measured in this run."""
    f = line.get("forms", {})
    out = {"fp64_solve_p50_ms": line["latency_ms"]["p50"], "fp64_solve_p99_ms": line["latency_ms"]["p99"]}

    def pick(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return float(f"{d:.6g}") if isinstance(d, float) else d

    out["batched_solves_per_s"] = pick(f, "batched", "solves_per_s")
    out["batched_vs_plain_fp64"] = pick(f, "batched", "speedup_vs_plain_fp64")
    out["batched_e2e_solves_per_s"] = pick(f, "batched", "e2e_solves_per_s")
    for mode in ("device_resident", "host_inputs"):
        for prec in ("mixed", "mixed_adaptive", "fp64"):
            out[f"serving_{mode}_{prec}_solves_per_s"] = pick(f, "serving", mode, prec, "solves_per_s")
            out[f"serving_{mode}_{prec}_p99_ms"] = pick(f, "serving", mode, prec, "p99_ms")
    pts = pick(f, "serving_stream", "points") or []
    for pt in pts:
        r = int(pt["rate_hz"])
        for prec in ("mixed", "mixed_adaptive", "fp64"):
            out[f"stream_{r}hz_{prec}_poisson_p50_ms"] = pick(pt, prec, "poisson_p50_ms")
            out[f"stream_{r}hz_{prec}_p99_ms"] = pick(pt, prec, "p99_ms")
    out["convdiff513_fp64_ms"] = pick(f, "convdiff", "fp64", "ms")
    out["convdiff513_mixed_ms"] = pick(f, "convdiff", "mixed", "ms")
    out["convdiff513_mixed_rel_l2_vs_gpu_fp64"] = pick(f, "convdiff", "mixed", "rel_l2_vs_fp64")
    out["convdiff129_mixed_rel_l2_vs_fp64_oracle"] = pick(f, "convdiff", "vs_fp64_oracle", "mixed", "rel_l2_vs_oracle")
    out["convdiff129_fp64_rel_l2_vs_fp64_oracle"] = pick(f, "convdiff", "vs_fp64_oracle", "fp64", "rel_l2_vs_oracle")
    for k in ("config1_cg_129", "config1_jacobi_129", "projection_256"):
        out[f"{k}_gpu_e2e_ms"] = pick(f, "reference_code", k, "gpu_e2e_ms")
        out[f"{k}_reference_cpu_ms"] = pick(f, "reference_code", k, "cpu_ms")
        out[f"{k}_rel_l2_vs_reference"] = pick(f, "reference_code", k, "rel_l2_vs_reference")
    out["vtk_legacy_ms"] = pick(f, "output", "vtk_legacy", "ms")
    out["cpu_baseline_solves_per_s"] = pick(line, "cpu_baseline", "value")
    return out


def _pct(xs, q):
    """Nearest-rank percentile."""
    xs = sorted(xs)
    if not xs:
        return None
    return xs[min(len(xs) - 1, max(0, math.ceil(q / 100.0 * len(xs)) - 1))]


def bench_serving_stream(abi, rates=(50.0, 100.0, 200.0), count=64, seed=11):
    """Serving stream with a seeded rate sweep: at each rate, `count` requests
    with Poisson-process arrivals, each submitted at its arrival time, mixing
    Poisson solves (60 %: 2D sides 65..513, 3D sides 65..129, tol 1e-10),
    200-step explicit heat runs (25 %: 2D sides 65..257, dt 0.9x the
    forward-Euler limit) and 2D pressure projections (15 %: 256^2..1024^2,
    CG to 1e-10); host inputs and outputs. Per rate and precision: completed
    requests/s over the run, p50/p99 latency (arrival -> result in host
    memory) over all requests and over the Poisson requests alone, and the
    peak HBM the server held."""
    from pde_solver_b200 import synthetic
    from pde_solver_b200.server import Server

    points = []
    for rate in rates:
        items = []
        for t, kind, sp in synthetic.serving_requests(count, seed=seed, rate_hz=rate):
            if kind == "poisson":
                items.append((t, kind, synthetic.poisson_request_problem(sp["n"], sp["dim"], sp["seed"])))
            elif kind == "heat":
                items.append((t, kind, synthetic.heat_problem(sp["n"])))
            else:
                u, v, p0 = synthetic.projection_fields(sp["n"], sp["seed"])
                items.append((t, kind, (u, v, p0, sp["n"])))
        kinds = {k: sum(1 for _, kk, _ in items if kk == k) for k in ("poisson", "heat", "projection")}
        point = {"rate_hz": rate, "requests": count, "kinds": kinds, "span_s": items[-1][0]}
        # mixed: every Poisson request batched; mixed_adaptive: while fewer than
        # 8 Poisson requests wait, each runs single-grid mixed on a free lane
        for name, prec, lanes, single in (("mixed", abi.MIXED, 6, 0), ("mixed_adaptive", abi.MIXED, 6, 8),
                                          ("fp64", abi.FP64, 16, 0)):
            with Server(lanes=lanes, max_batch=64, precision=prec, single_below=single, tile_x=64, tile_y=64,
                        tile_z=32, pre_smooth=1, post_smooth=2, inner_tol=1e-5) as s:

                def submit(kind, x):
                    if kind == "poisson":
                        return s.submit_poisson(x)
                    if kind == "heat":
                        return s.submit_heat(x[0], x[1], 200)
                    u, v, p0, n = x
                    h = 1.0 / (n - 1)
                    return s.submit_projection(u, v, None, p0, n, n, 1, h, h, 1.0, 0.01)

                # one request of each kind before the clock starts
                for kind in ("poisson", "heat", "projection"):
                    first = next((x for _, kk, x in items if kk == kind), None)
                    if first is not None:
                        s.wait(submit(kind, first))
                s.stats(reset=True)
                ids = []
                t0 = time.perf_counter()
                for t, kind, x in items:
                    delay = t0 + t - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                    ids.append((kind, submit(kind, x)))
                res = [(kind, s.wait(i)[1]) for kind, i in ids]
                wall = time.perf_counter() - t0
                st = s.stats()
            pl = [r.latency_ms for kind, r in res if kind == "poisson"]
            point[name] = {"requests_per_s": count / wall, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                           "poisson_p50_ms": _pct(pl, 50), "poisson_p99_ms": _pct(pl, 99),
                           "failed": int(sum(r.status != abi.OK for _, r in res)),
                           "max_group": int(max(r.group_size for _, r in res)),
                           "hbm_peak_gb": st.bytes_peak / 1e9, "lanes": lanes, "single_below": single}
        points.append(point)
    return {"workload": f"seeded Poisson-process arrivals at {', '.join(f'{r:g}' for r in rates)} requests/s, "
                        f"{count} requests each: Poisson 60 % / heat 25 % / projection 15 %, host inputs",
            "points": points}


def run_reference(args):
    """The CPU implementation of the headline workload on the host cores: each
    step is one whole converged 257^3 solve by the oracle port of the same
    MG-PCG (oracle/restate.c; the reference's CPU path has no 3D divergence-form
    solver), W warm-up solves then exactly K timed ones."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from pde_solver_b200 import synthetic

    prob = synthetic.varcoef_poisson_3d(args.n, seed=SEED)
    if args.warmup > 0:
        cpu_solve_times(prob, args.warmup)
    times, iters, cores = cpu_solve_times(prob, args.steps)
    total = sum(times)
    value = args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": config(args.n, "cpu"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": (f"oracle/restate.c MG-PCG (the reference's CPU path has no 3D "
                                    f"divergence-form MG-PCG), {cores} OpenMP threads; each step one whole "
                                    f"converged solve ({iters} iterations)")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "latency_ms": {"p50": 1e3 * _pct(times, 50), "p99": 1e3 * _pct(times, 99)},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU side

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    from pde_solver_b200 import abi, synthetic
    from pde_solver_b200.problem import default_options

    from pde_solver_b200 import replicas

    world, rank, local = replicas.rank_env()
    if world > 1:
        torch.cuda.set_device(local)
    dist = replicas.init("nccl", timeout_s=600)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    lib = abi.load()

    n = args.n
    prob = synthetic.varcoef_poisson_3d(n, seed=replicas.replica_seed(SEED, rank))
    N = prob.n
    opt = default_options(method=abi.MG_PCG, tol=1e-10, tol_mode=abi.TOL_RELATIVE, max_iter=400, device=local)
    stream = torch.cuda.current_stream(device)
    assert lib.pdeb200_set_stream(local, C.c_void_p(stream.cuda_stream)) == abi.OK

    # ---- device-resident inputs
    k_dev = torch.from_numpy(prob.k).to(device)
    f_dev = torch.from_numpy(prob.f).to(device)
    out_dev = torch.empty(N, dtype=torch.float64, device=device)
    import copy

    dprob = copy.copy(prob)
    dprob.k, dprob.f = None, None
    dprob.mem_space = abi.MEM_DEVICE
    dprob.k_dev, dprob.f_dev = k_dev.data_ptr(), f_dev.data_ptr()
    cdev = dprob.to_c()

    def solve_dev():
        rep = abi.Report()
        st = lib.pdeb200_solve(C.byref(cdev), C.byref(opt), C.c_void_p(out_dev.data_ptr()), C.byref(rep))
        if st != abi.OK:
            raise RuntimeError(f"solve failed: {st} {rep.message.decode()}")
        return rep

    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        rep = solve_dev()
    iters = rep.iterations
    rel = rep.rel_residual

    def barrier():
        if dist is not None:
            dist.barrier()

    launches = 0
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_dev, step_wall = [], []
    e0.record(stream)
    for _ in range(args.steps):
        t_step = time.perf_counter()
        rep = solve_dev()
        step_wall.append((time.perf_counter() - t_step) * 1e3)
        step_dev.append(rep.device_ms)
        launches += rep.kernel_launches
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    latency = {"p50": _pct(step_dev, 50), "p99": _pct(step_dev, 99), "max": max(step_dev),
               "over": "device time of each timed solve"}
    ms = replicas.max_over_ranks(ms, dist, device)
    value = replicas.aggregate_rate(world, args.steps, ms)

    # ---- end to end through the same C-ABI call with pinned host buffers
    k_host = torch.from_numpy(prob.k).pin_memory()
    f_host = torch.from_numpy(prob.f).pin_memory()
    out_host = torch.empty(N, dtype=torch.float64).pin_memory()
    hprob = copy.copy(prob)
    hprob.k, hprob.f = None, None
    ch = hprob.to_c()
    ch.k = C.cast(C.c_void_p(k_host.data_ptr()), C.POINTER(C.c_double))
    ch.f = C.cast(C.c_void_p(f_host.data_ptr()), C.POINTER(C.c_double))

    def solve_host():
        rep = abi.Report()
        st = lib.pdeb200_solve(C.byref(ch), C.byref(opt), C.c_void_p(out_host.data_ptr()), C.byref(rep))
        if st != abi.OK:
            raise RuntimeError(f"solve failed: {st} {rep.message.decode()}")
        return rep

    solve_host()
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        solve_host()
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = e2.elapsed_time(e3)
    ms_e2e = replicas.max_over_ranks(ms_e2e, dist, device)
    e2e_value = replicas.aggregate_rate(world, args.steps, ms_e2e)
    ok_host = np.allclose(out_host.numpy(), out_dev.cpu().numpy(), rtol=0, atol=1e-12 * float(out_dev.abs().max()))

    # ---- live per-kernel roofline (events around each finest-level launch)
    lib.pdeb200_profile_enable(local, 1)
    for _ in range(2):
        solve_dev()
    stats = (abi.KernelStat * 128)()
    cnt = lib.pdeb200_profile_read(local, stats, 128)
    lib.pdeb200_profile_enable(local, 0)
    kern = []
    for q in range(min(cnt, 128)):
        s = stats[q]
        if s.launches:
            kern.append({"name": s.name.decode(), "launches": int(s.launches), "total_ms": s.total_ms,
                         "avg_us": 1e3 * s.total_ms / s.launches, "bytes": s.bytes_per_launch,
                         "gbs": s.bytes_per_launch / (s.total_ms / s.launches / 1e3) / 1e9})
    kern.sort(key=lambda d: -d["total_ms"])
    fine = [d for d in kern if d["name"].endswith("@L0")]
    peak, peak_kind = peaks()
    top = fine[0] if fine else (kern[0] if kern else None)
    roofline = None
    if top:
        traffic = ncu_traffic(top["name"])
        roofline = {"bound": "hbm", "kernel": top["name"], "achieved": round(top["gbs"], 1), "peak": peak,
                    "unit": "GB/s", "frac": round(top["gbs"] / peak, 4), "peak_source": peak_kind,
                    "traffic": traffic, "algorithmic_bytes_per_launch": top["bytes"],
                    "avg_launch_us": round(top["avg_us"], 2),
                    "kernels": [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in d.items()}
                                for d in kern[:16]]}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded, generated on the host)",
        "config": config(n, "inputs larger than L2 (k, f, x, r, p, q: 136 MB each)"),
        "iterations": iters, "rel_residual": rel, "dof_iterations_per_s": N * iters * value, "latency_ms": latency,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * N * 8, "d2h_bytes_per_step": N * 8,
                "matches_device_result": bool(ok_host)},
        "gpu_launches": launches, "clocks": clocks, "roofline": roofline,
        # each timed solve: its own device time (events inside the call) and
        # the host wall time of the call
        "steps_detail": {"device_ms": [round(v, 3) for v in step_dev], "wall_ms": [round(v, 3) for v in step_wall]},
    }
    if rank == 0 and world == 1 and not args.no_forms:
        forms = {}
        for key, run in (("batched", lambda: bench_batched(lib, abi)), ("serving", lambda: bench_serving(abi)),
                         ("serving_stream", lambda: bench_serving_stream(abi)),
                         ("output", lambda: bench_output(out_dev, n)),
                         ("convdiff", lambda: bench_convdiff(lib, abi, device)),
                         ("reference_code", lambda: reference_code_paths(lib, abi, device))):
            try:
                forms[key] = run()
            except Exception as exc:  # the forms never block the headline line
                forms[key] = {"error": str(exc)}
        line["forms"] = forms
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_sample(prob)
        except Exception as exc:  # the baseline never blocks the GPU line
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {exc}"}
    if "forms" in line:
        # the forms' headline figures, last in the line so a kept tail holds them
        line["summary"] = summarize(line)
    lib.pdeb200_set_stream(local, None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
