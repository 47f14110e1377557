#!/usr/bin/env python
"""DOF-solves/s at a 1e-8 relative residual: PCG with the multigrid preconditioner, mixed
precision (FP32 V-cycle inside FP64 flexible CG) against the plain FP64 form, on one B200.

Workload: P1 heat conduction in the unit cube of 128^3 cells split into 6 Kuhn tetrahedra
(2,146,689 points, 2,113,407 free unknowns, 31.8M entries), conductivity exp(N(0, 1)) per
tetrahedron (numpy PCG64 seed 1234), T = 1 on x = 0 and T = 0 on x = 1, source 1.0. A step is
1 solve of 1 right side from x = 0 to |b - A x| / |b| <= 1e-8 (the true FP64 residual is
checked and reported). The operator and its hierarchy stay resident (the reference's `Solver`
is made once and solves many right sides).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs under torchrun, one independent replica per GPU (the path does not shard); the
timed region of each rank is bracketed by a barrier and CUDA events on the solver's own
stream, and the slowest rank's time gives the whole-job figure.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 128
TOL = 1e-8
SEED = 1234
METRIC = "DOF-solves/s at 1e-8 rel. residual, mixed vs FP64 PCG-MG; p50/p99 latency"
UNIT = "DOF-solves/s"


def args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cells", type=int, default=N_CELLS)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile", action="store_true",
                   help="only the timed mixed-precision solves (the command profiled by ncu)")
    p.add_argument("--format", type=int, default=0, help="0: stencil where possible, 1: SELL")
    p.add_argument("--breakdown", action="store_true",
                   help="print each solver's levels and the device time of each kernel of 1 "
                        "PCG iteration (kernels launched one by one), then exit")
    p.add_argument("--graph", type=int, default=0,
                   help="0/1: the PCG loop as 1 CUDA graph; 2: kernels launched one by one (so "
                        "that a profiler lists each kernel of the loop)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ------------------------------------------------------------------ clocks during the timed run
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.file,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ the problem
def build_problem(cells):
    from femahoy_b200 import meshgen as mg
    return mg.heat_cube(cells, seed=SEED)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary (if any)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------ CPU baseline (oracle)
def oracle_solve_rate(A, rhs, planes, pts, comp, budget_s=60.0):
    """The oracle's PCG with the reference's line Gauss-Seidel multigrid (FP64, 1 thread) on
    the same system: (DOF-solves/s, iterations, solve seconds, setup seconds)."""
    import oracle
    ptr, idx, val = A.arrays()
    Ao = oracle.Csr.from_arrays(A.n, ptr, idx, val)
    t0 = time.perf_counter()
    so = oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, it, res = so.solve(rhs, tol=TOL)
    solve = time.perf_counter() - t0
    return A.n / solve, it, solve, setup, res


def run_reference(opt, rank, world):
    """The reference arm: the oracle restatement of the reference's CPU path (assembly, the
    Galerkin hierarchy with line Gauss-Seidel, PCG) on the host, rank 0 only."""
    if rank != 0:
        return
    import oracle
    from femahoy_b200 import meshgen as mg
    t0 = time.perf_counter()
    h = build_problem(opt.cells)
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(0, h.xyz, h.nodes, h.coef)
    a = k.submatrix(h.free)
    rhs = k.reduced_rhs(h.load, h.values, h.free)
    assemble_s = time.perf_counter() - t0
    planes, pts, comp = mg.grid_unknowns(h)
    t0 = time.perf_counter()
    so = oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    setup_s = time.perf_counter() - t0
    # A step is 1 full solve when it fits the budget, else a bounded run of PCG iterations
    # scaled by the iterations of the full solve of the warm-up.
    t0 = time.perf_counter()
    _, iters, res = so.solve(rhs, tol=TOL)
    full = time.perf_counter() - t0
    per_it = full / max(iters, 1)
    budget = 150.0 / max(1, opt.steps + opt.warmup)
    sample_its = iters if full <= budget else max(1, int(budget / per_it))
    times = []
    for step in range(max(0, opt.warmup - 1) + opt.steps):
        t0 = time.perf_counter()
        if sample_its >= iters:
            so.solve(rhs, tol=TOL)
            dt = time.perf_counter() - t0
        else:
            try:
                so.solve(rhs, tol=TOL, max_iter=sample_its)
            except oracle.OracleError:
                pass
            dt = (time.perf_counter() - t0) * iters / sample_its
        if step >= max(0, opt.warmup - 1):
            times.append(dt)
    value = a.n * len(times) / sum(times)
    sample = (f"full solves of the {opt.cells}^3 system ({iters} PCG iterations)"
              if sample_its >= iters else
              f"{sample_its} of the {iters} PCG iterations of the {opt.cells}^3 solve per step, "
              f"scaled to 1 solve")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": len(times), "warmup": opt.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"P1 heat, {opt.cells}^3 Kuhn box, lognormal k (seed {SEED}), "
                               f"1 RHS to 1e-8", "free_dofs": a.n, "tol": TOL,
                   "precision": "fp64 (reference algorithm: PCG + line Gauss-Seidel MG)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_detail": {"iterations": iters, "residual": res, "assembly_s": assemble_s,
                             "setup_s": setup_s, "full_solve_s": full,
                             "host_cores": os.cpu_count(),
                             "note": "the reference is single-threaded (no threads in fh-fem)"},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def run_ours(opt, rank, world, local):
    import torch
    import torch.distributed as dist

    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    h = build_problem(opt.cells)
    lib = fg.lib()
    t0 = time.perf_counter()
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    assemble_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    A = K.submatrix(h.free)
    rhs = fg.reduced_rhs(K, h.load, h.values, h.free)
    reduce_s = time.perf_counter() - t0
    n_free = A.n
    del K
    planes, pts, comp = mg.grid_unknowns(h)
    unknowns = fg.Unknowns.Grid(fg.Level(planes, pts, comp))

    def make(precision):
        t = time.perf_counter()
        s = fg.Solver(A, unknowns, fg.Method.Multigrid,
                      options=fg.Options(precision=precision, format=opt.format,
                                         graph=opt.graph)).with_tol(TOL)
        return s, time.perf_counter() - t

    b = torch.from_numpy(rhs).cuda()
    x = torch.zeros_like(b)

    def timed(solver, steps, warmup, clocks=None):
        stream = torch.cuda.ExternalStream(lib.femgpu_solver_stream(solver.handle))
        for _ in range(warmup):
            with torch.cuda.stream(stream):
                x.zero_()
            solver.solve_device(b.data_ptr(), x.data_ptr())
        barrier()
        stream.synchronize()
        if clocks:
            clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lat, its, launches, res = [], [], 0, []
        e0.record(stream)
        for _ in range(steps):
            with torch.cuda.stream(stream):
                x.zero_()
            st = solver.solve_device(b.data_ptr(), x.data_ptr())
            lat.append(st.seconds)
            its.append(st.iterations)
            res.append(st.true_residual)
            launches += st.launches + 1
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop() if clocks else None
        ms = e0.elapsed_time(e1)
        return ms, lat, its, launches, res, clk

    if opt.breakdown:
        for precision in (fg.MIXED, fg.FP64):
            s, _ = make(precision)
            for _ in range(3):
                with torch.cuda.stream(torch.cuda.ExternalStream(
                        lib.femgpu_solver_stream(s.handle))):
                    x.zero_()
                st = s.solve_device(b.data_ptr(), x.data_ptr())
            if rank == 0:
                print(f"== {'mixed' if precision == fg.MIXED else 'fp64'}: {st.iterations} "
                      f"iterations, {st.seconds * 1e3:.3f} ms per solve (CUDA graph)")
                print(s.describe())
                print(s.breakdown(), flush=True)
            del s
        return
    mixed, setup_mixed = make(fg.MIXED)
    clocks = Clocks(torch.cuda.current_device())
    ms, lat, its, launches, res, clk = timed(mixed, opt.steps, opt.warmup, clocks)
    ms_max = max_over_ranks(ms)
    value = world * n_free * opt.steps / (ms_max / 1e3)
    if opt.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "value": value, "unit": UNIT,
                              "ms_per_step": ms_max / opt.steps, "iterations": its,
                              "launches": launches, "true_residual": max(res)}), flush=True)
        return

    # The dominant kernel alone: the finest FP32 Chebyshev step (SpMV + smoother update).
    kms, kbytes = ctypes.c_double(), ctypes.c_double()
    fg._lib.check(lib.femgpu_solver_kernel_time(mixed.handle, 0, 50, ctypes.byref(kms),
                                                ctypes.byref(kbytes)))
    peak, peak_kind = measured_peak()
    achieved = kbytes.value / (kms.value * 1e-3) / 1e9
    traffic = profiled_traffic()

    # e2e: the same solve through the host C ABI from pinned host memory (copies inside).
    hb = torch.from_numpy(rhs).pin_memory()
    hx = torch.zeros(n_free, dtype=torch.float64).pin_memory()
    stream = torch.cuda.ExternalStream(lib.femgpu_solver_stream(mixed.handle))
    st_ = fg._lib.Stats_t()
    for _ in range(opt.warmup):
        hx.zero_()
        fg._lib.check(lib.femgpu_solver_solve(mixed.handle, ctypes.c_void_p(hb.data_ptr()),
                                              ctypes.c_void_p(hx.data_ptr()), None,
                                              ctypes.byref(st_)))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(opt.steps):
        hx.zero_()
        fg._lib.check(lib.femgpu_solver_solve(mixed.handle, ctypes.c_void_p(hb.data_ptr()),
                                              ctypes.c_void_p(hx.data_ptr()), None,
                                              ctypes.byref(st_)))
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = world * n_free * opt.steps / (e2e_ms / 1e3)
    mixed_bytes = mixed.device_bytes()
    levels = mixed.levels()
    del mixed

    # The plain FP64 form on the same workload.
    plain, setup_fp64 = make(fg.FP64)
    ms64, lat64, its64, _, res64, _ = timed(plain, opt.steps, opt.warmup)
    ms64 = max_over_ranks(ms64)
    value64 = world * n_free * opt.steps / (ms64 / 1e3)
    del plain

    cpu = None
    if rank == 0 and world == 1 and not opt.no_cpu_baseline:
        try:
            rate, cit, csolve, csetup, cres = oracle_solve_rate(A, rhs, planes, pts, comp)
            cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"1 full solve of the same {opt.cells}^3 system by the oracle "
                             f"(reference algorithm: FP64 PCG + line Gauss-Seidel MG), "
                             f"{cit} iterations, {csolve:.1f} s (setup {csetup:.1f} s "
                             f"excluded)"}
        except Exception as e:  # the baseline is reported, never the product
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"failed: {e}"}

    lat_ms = np.array(lat) * 1e3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": opt.steps,
        "warmup": opt.warmup, "ms_per_step": ms_max / opt.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 outer",
        "data": "synthetic",
        "config": {
            "workload": f"P1 heat, {opt.cells}^3 Kuhn box (6 tets/hex), lognormal k seed {SEED}, "
                        f"1 RHS to 1e-8, mixed precision PCG-MG",
            "free_dofs": n_free, "tol": TOL, "levels": levels,
            "flush": "inputs larger than L2 (the FP64 operator alone is 0.4 GB)",
            "parallelism": f"replicas x{world}",
        },
        "latency_ms": {"p50": float(np.percentile(lat_ms, 50)),
                       "p99": float(np.percentile(lat_ms, 99))},
        "iterations": {"mixed": int(np.median(its)), "fp64": int(np.median(its64))},
        "true_residual": {"mixed": float(max(res)), "fp64": float(max(res64))},
        "fp64": {"value": value64, "unit": UNIT, "ms_per_step": ms64 / opt.steps,
                 "p50_ms": float(np.percentile(np.array(lat64) * 1e3, 50)),
                 "p99_ms": float(np.percentile(np.array(lat64) * 1e3, 99))},
        "mixed_over_fp64": value / value64,
        "setup_s": {"assembly": assemble_s, "submatrix_and_rhs": reduce_s,
                    "solver_mixed": setup_mixed, "solver_fp64": setup_fp64},
        "including_setup": world * n_free / (assemble_s + reduce_s + setup_mixed
                                             + ms_max / opt.steps / 1e3),
        "device_bytes": mixed_bytes,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": "k_cheb_step<float> (finest level)",
                     "bytes_per_launch": kbytes.value, "launch_ms": kms.value,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * n_free,
                "d2h_bytes_per_step": 8 * n_free},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    opt = args()
    rank, world, local = dist_env()
    if opt.impl == "reference":
        run_reference(opt, rank, world)
        return
    run_ours(opt, rank, world, local)


if __name__ == "__main__":
    main()
