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
    p.add_argument("--tail", type=int, default=0,
                   help="> 0: levels of at most this many rows run as 1 fused cooperative "
                        "kernel (0: none, the default)")
    p.add_argument("--launch", type=int, default=0,
                   help="0: programmatic dependent launch in the PCG loop (default), 1: plain")
    p.add_argument("--lower", type=float, default=0.0,
                   help="Chebyshev interval's lower end as a fraction of lambda_max (0: 0.3)")
    p.add_argument("--coarsest", type=int, default=0,
                   help="the largest level the dense coarse solve takes (0: 3000, the reference's)")
    p.add_argument("--stencil", type=int, default=0,
                   help="stencil product kernel: 0 tuned, 1 runtime K, 2 compile-time K, "
                        "3 2 rows per thread, 4 marching planes")
    p.add_argument("--smoother", type=int, default=0,
                   help="Chebyshev smoother polynomial: 0/1 first kind, 4 fourth kind")
    p.add_argument("--cluster", type=int, default=0,
                   help="small levels: 1 each leg as 1 cluster launch, 0 a launch per step")
    p.add_argument("--upper", type=float, default=0.0,
                   help="Chebyshev interval upper end over lambda_max (0: 1.1)")
    p.add_argument("--l2", type=int, default=0,
                   help="1: the coarsest inverse persisting in L2")
    p.add_argument("--tiles", type=int, default=0,
                   help="finest FP32 stencil steps from bulk-copied tiles: 0 tuned, 1 off, 2 on")
    p.add_argument("--values", type=int, default=0,
                   help="mixed form's stencil levels: 0 default, 1 FP32, 2 FP16 coefficients")
    p.add_argument("--degree", type=int, default=0,
                   help="Chebyshev degree of each pre- and post-smoothing (0: the default, 2)")
    p.add_argument("--breakdown", action="store_true",
                   help="print each solver's levels and the device time of each kernel of 1 "
                        "PCG iteration (kernels launched one by one), then exit")
    p.add_argument("--workload", default="heat",
                   choices=["heat", "cantilever", "p2beam", "batch", "serve", "stream",
                            "recover", "transient", "modes", "hexheat", "hexbeam",
                            "hexrecover", "hexmodes", "prism", "direct"],
                   help="heat: 1 right side of the 128^3 heat cube (the headline line); "
                        "cantilever: the 40x4x4 P1 cantilever at 1e-10; p2beam: the 200x20x20 "
                        "P2 beam; batch: 256 cantilevers x 16 load cases in 1 batched solve; "
                        "serve: a Poisson stream of solve requests through the server; "
                        "stream: a Poisson stream of single load cases of the 256 batched "
                        "cantilevers, admitted into the running device loop (continuous "
                        "batching); "
                        "recover: the stress recovery of the solved 200x20x20 P2 beam; "
                        "transient: backward-Euler steps of the 128^3 heat cube; "
                        "modes: 10 lowest modes of a 100x10x10 P2 beam; hexheat: the 128^3 "
                        "heat cube on box cells; hexbeam: a cantilever of 256x32x32 box cells "
                        "with incompatible modes (2 materials); hexrecover: the stress "
                        "recovery of that cantilever; hexmodes: 10 modes of a 128x16x16 "
                        "box-cell cantilever")
    p.add_argument("--by-cells", action="store_true",
                   help="hexbeam: the coarse matrices from the cells, as the reference forms "
                        "them (default: Galerkin products, fewer iterations here)")
    p.add_argument("--systems", type=int, default=256, help="batch: cantilevers in the batch")
    p.add_argument("--prism-cell", type=float, default=0.04,
                   help="prism: max_cell of the prism mesh (grid.rs Spacing)")
    p.add_argument("--rates", default="10,50,200,500",
                   help="serve: Poisson arrival rates (requests/s) to replay the stream at")
    p.add_argument("--requests", type=int, default=40, help="serve: requests per rate")
    p.add_argument("--builders", type=int, default=3,
                   help="serve: threads that build new meshes' solvers side by side")
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
        """Starts the sampler and returns once it has written its first sample (at most 15 s):
        nvidia-smi's own start-up then lies outside the timed region."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.file,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 15.0 and self.proc.poll() is None:
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.05)

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


def build_system(opt):
    """The device system of a single-solver workload: (A, rhs, unknowns, facts). `facts` holds
    the workload's text, tolerance, assembly and reduction seconds, and a maker of the oracle's
    solver for the CPU baseline (reference algorithm, FP64)."""
    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg
    import oracle
    if opt.workload == "cantilever":
        prob = mg.cantilever_p1()
        kind, tol = fg.P1_ELASTIC, 1e-10
        text = ("P1 elasticity cantilever 100x10x10 mm as 40x4x4 hexes x 6 Kuhn tets (3,000 free "
                "unknowns), E 210 GPa, nu 0.3, clamped at x = 0, 1 MPa on the top face, to 1e-10, "
                "FP64 and mixed PCG-MG")
    elif opt.workload == "hexheat":
        prob = mg.heat_cube_hex(opt.cells, seed=SEED)
        kind, tol = fg.HEX8_HEAT, TOL
        text = (f"P1 heat on box cells (the reference's box-grid model), {opt.cells}^3 hex "
                f"cells of the unit cube, lognormal k seed {SEED}, 1 RHS to 1e-8, mixed "
                f"precision PCG-MG")
    elif opt.workload == "hexbeam":
        nx, ny = 2 * opt.cells, max(1, opt.cells // 4)
        prob = mg.hex_cantilever(nx=nx, ny=ny, nz=ny, length=8.0, width=1.0, depth=1.0,
                                 e=1000.0, nu=0.3, load=-1.0, seed=SEED)
        kind, tol = fg.HEX8_ELASTIC, TOL
        text = (f"elasticity on box cells with incompatible modes (the reference's box-grid "
                f"elastic model), a {nx}x{ny}x{ny} cell cantilever 8x1x1, isotropic (E 1000, nu "
                f"0.3) and orthotropic cells (seed {SEED}), clamped at x = 0, a tip load, 1 RHS "
                f"to 1e-8, mixed precision PCG-MG, coarse matrices "
                f"{'from the cells' if opt.by_cells else 'by Galerkin products'}")
    elif opt.workload == "p2beam":
        box = mg.box(200, 20, 20, (200.0, 20.0, 20.0))
        q = fg.Quadratic.new(box.points, box.tets)
        prob = mg.beam_p2(q.edges, q.tets, mesh=box, seed=SEED)
        kind, tol = fg.P2_ELASTIC, TOL
        text = (f"P2 elasticity box beam 200x20x20 mm as 200x20x20 hexes x 6 Kuhn tets (10-node), "
                f"E 70 GPa, nu 0.33, clamped at x = 0, random traction on x = L (seed {SEED}), "
                f"p-multigrid P2 -> P1 then geometric levels, to 1e-8")
    else:
        prob = build_problem(opt.cells)
        kind, tol = fg.P1_HEAT, TOL
        text = heat_text(opt.cells)
    t0 = time.perf_counter()
    K = fg.Csr.assemble(kind, prob.xyz, prob.nodes, prob.coef)
    assemble_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    reduce_s = time.perf_counter() - t0
    del K
    if opt.workload == "p2beam":
        P, coarse = fg.prolongation(prob.xyz, box.n, q.edges, prob.free)
        unknowns = fg.Unknowns.Quadratic(prob.xyz[prob.free // 3], P, coarse)

        def oracle_solver(Ao):
            Po = oracle.Rect.from_arrays(P.rows, P.cols, P.ptr, P.idx, P.val)
            return oracle.Solver(Ao, "quadratic", xyz=prob.xyz[prob.free // 3], p=Po,
                                 coarse=coarse, method="multigrid")
    else:
        planes, pts, comp = mg.grid_unknowns(prob)
        unknowns = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
        cells = None
        if opt.workload == "hexbeam" and opt.by_cells:
            # elastic.rs:518-537: the coarse matrices from the cells, as the reference solves
            # its box-grid elastic models.
            t0 = time.perf_counter()
            origin, cls, keys = mg.hex_classes(prob)
            cells = fg.Cells(origin, cls, fg.hex_elements(keys))
            assemble_s += time.perf_counter() - t0

        def oracle_solver(Ao):
            oc = None if cells is None else (cells.origin, cells.cls, cells.matrices)
            return oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp,
                                 method="multigrid", cells=oc)
    facts = {"text": text, "tol": tol, "assemble_s": assemble_s, "reduce_s": reduce_s,
             "oracle_solver": oracle_solver, "cells": cells if opt.workload != "p2beam" else None,
             "direct_xyz": prob.xyz[prob.free // prob.comps]}
    return A, rhs, unknowns, facts


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary (if any)."""
    path = os.path.join(ROOT, "profiles", "k_cheb_step_heat128_level0.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------ CPU baseline (oracle)
def oracle_solve_rate(A, rhs, make_solver, tol, direct_xyz=None):
    """The oracle's PCG with the reference's multigrid (FP64) on the same system, on 1 thread
    (the reference's) and then on all host cores (its matrix products and dot products split
    across threads; the smoothers stay sequential, as the reference's are). Returns a dict:
    rate, iterations, solve / setup seconds, residual, all-cores rate and cores, and the
    solutions the device's are checked against: `x_tol` (the oracle's PCG-MG at the same
    tolerance), `x_tight` (its PCG-MG continued from x_tol to 1e-12 on all cores) and, for
    systems of at most 40,000 unknowns with `direct_xyz`, `x_direct` (its multifrontal
    Cholesky, cholesky.rs:44-167)."""
    import oracle
    ptr, idx, val = A.arrays()
    Ao = oracle.Csr.from_arrays(A.n, ptr, idx, val)
    t0 = time.perf_counter()
    so = make_solver(Ao)
    setup = time.perf_counter() - t0
    oracle.set_threads(1)
    t0 = time.perf_counter()
    x_tol, it, res = so.solve(rhs, tol=tol)
    solve = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    try:
        t0 = time.perf_counter()
        so.solve(rhs, tol=tol)
        solve_all = time.perf_counter() - t0
        x_tight, _, res_tight = so.solve(rhs, x=x_tol, tol=min(tol, 1e-12))
    finally:
        oracle.set_threads(1)
    out = {"rate": A.n / solve, "iterations": it, "solve_s": solve, "setup_s": setup,
           "residual": res, "rate_all": A.n / solve_all, "cores": cores, "x_tol": x_tol,
           "x_tight": x_tight, "residual_tight": res_tight, "x_direct": None}
    if direct_xyz is not None and A.n <= 40000:
        out["x_direct"], _ = oracle.direct_solve(Ao, direct_xyz, rhs)
    return out


def setup_phases(solver):
    """The solver's own setup timers (seconds per phase, host clock until the phase's device work
    finished), from the "setup seconds:" line of its description."""
    for line in solver.describe().splitlines():
        if line.startswith("setup seconds:"):
            out = {}
            for part in line[len("setup seconds:"):].split(";"):
                name, _, sec = part.strip().rpartition(" ")
                if name:
                    out[name] = float(sec)
            return out
    return {}


def error_vs_oracle(x, ref):
    """|x - x_oracle|_2 / |x_oracle|_2 against each oracle solution of `oracle_solve_rate`."""
    def rel(y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))
    out = {"vs_oracle_pcg_mg_same_tol": rel(ref["x_tol"]),
           "vs_oracle_pcg_mg_1e-12": rel(ref["x_tight"])}
    if ref.get("x_direct") is not None:
        out["vs_oracle_direct"] = rel(ref["x_direct"])
    return out


def heat_text(cells):
    return (f"P1 heat, {cells}^3 Kuhn box (6 tets/hex), lognormal k seed {SEED}, 1 RHS "
            f"to 1e-8")


def workload_config(text, n_free, nnz, tol, world):
    """The `config` of a single-solver line, the same in both arms: the workload, its size and
    tolerance, whether its operator alone exceeds the 126 MB L2 (FP32 values and int32
    columns), and the replicas."""
    big = nnz * 8 > (126 << 20)
    return {"workload": text, "free_dofs": int(n_free), "tol": tol,
            "flush": ("inputs larger than L2" if big else
                      "none: the whole problem fits L2; launch- and latency-bound"),
            "parallelism": f"replicas x{world}"}


def run_reference(opt, rank, world):
    """The reference arm: the oracle restatement of the reference's CPU path (assembly, the
    Galerkin hierarchy with line Gauss-Seidel, PCG) on the host, rank 0 only, with every host
    thread it can use (the matrix and dot products; the smoothers stay sequential, as the
    reference's are). Each step, warm-up and timed alike, is 1 full solve of the system to the
    tolerance from x = 0."""
    if rank != 0:
        return
    import oracle
    from femahoy_b200 import meshgen as mg
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    t0 = time.perf_counter()
    h = build_problem(opt.cells)
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(0, h.xyz, h.nodes, h.coef)
    a = k.submatrix(h.free)
    rhs = k.reduced_rhs(h.load, h.values, h.free)
    nnz = len(a.arrays()[1])
    del k
    assemble_s = time.perf_counter() - t0
    planes, pts, comp = mg.grid_unknowns(h)
    t0 = time.perf_counter()
    so = oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    setup_s = time.perf_counter() - t0
    for _ in range(opt.warmup):
        so.solve(rhs, tol=TOL)
    times, iters, res = [], 0, None
    for _ in range(opt.steps):
        t0 = time.perf_counter()
        _, iters, res = so.solve(rhs, tol=TOL)
        times.append(time.perf_counter() - t0)
    value = a.n * len(times) / sum(times)
    sample = (f"1 full solve of the {opt.cells}^3 system per step ({iters} PCG iterations, "
              f"{np.mean(times):.2f} s), matrix and dot products on {cores} host threads")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": len(times), "warmup": opt.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(heat_text(opt.cells), a.n, nnz, TOL, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_detail": {"iterations": iters, "residual": res, "assembly_s": assemble_s,
                             "setup_s": setup_s, "host_cores": os.cpu_count(),
                             "precision": "fp64 (the reference's algorithm: PCG + line "
                                          "Gauss-Seidel multigrid)",
                             "note": "the reference itself is single-threaded (no threads in "
                                     "fh-fem); this arm runs its algorithm with the matrix and "
                                     "dot products on all host threads"},
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

    lib = fg.lib()
    A, rhs, unknowns, facts = build_system(opt)
    tol = facts["tol"]
    assemble_s, reduce_s = facts["assemble_s"], facts["reduce_s"]
    n_free = A.n
    nnz = A.shape[1]

    def make(precision):
        t = time.perf_counter()
        s = fg.Solver(A, unknowns, fg.Method.Multigrid, cells=facts["cells"],
                      options=fg.Options(precision=precision, format=opt.format,
                                         graph=opt.graph, tail=opt.tail,
                                         degree=opt.degree, launch=opt.launch,
                                         values=opt.values, tiles=opt.tiles,
                                         stencil=opt.stencil, l2=opt.l2,
                                         smoother=opt.smoother, cluster=opt.cluster,
                                         upper=opt.upper,
                                         coarsest=opt.coarsest,
                                         lower=opt.lower)).with_tol(tol)
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
    value = replica_value(world, n_free, opt.steps, ms_max)
    if opt.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "value": value, "unit": UNIT,
                              "ms_per_step": ms_max / opt.steps, "iterations": its,
                              "launches": launches, "true_residual": max(res)}), flush=True)
        return

    # The dominant kernel alone: the finest FP32 Chebyshev step (SpMV + smoother update). A
    # problem at or below the coarsest size (the cantilever) has no smoothing level: its solve
    # is the dense coarse product and a few PCG kernels, launch- and latency-bound.
    kms, kbytes = ctypes.c_double(), ctypes.c_double()
    roof_ok = lib.femgpu_solver_kernel_time(mixed.handle, 0, 50, ctypes.byref(kms),
                                            ctypes.byref(kbytes)) == 0
    peak, peak_kind = measured_peak()
    achieved = kbytes.value / (kms.value * 1e-3) / 1e9 if roof_ok else None
    traffic = profiled_traffic() if opt.workload == "heat" and opt.cells == N_CELLS else None

    # e2e: the same solve through the host C ABI from pinned host memory (copies inside), from
    # x = 0 as the reference's callers start it (femgpu_solver_solve_zero: b in, x out).
    hb = torch.from_numpy(rhs).pin_memory()
    hx = torch.zeros(n_free, dtype=torch.float64).pin_memory()
    stream = torch.cuda.ExternalStream(lib.femgpu_solver_stream(mixed.handle))
    st_ = fg._lib.Stats_t()
    for _ in range(opt.warmup):
        fg._lib.check(lib.femgpu_solver_solve_zero(mixed.handle, ctypes.c_void_p(hb.data_ptr()),
                                                   ctypes.c_void_p(hx.data_ptr()), None,
                                                   ctypes.byref(st_)))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(opt.steps):
        fg._lib.check(lib.femgpu_solver_solve_zero(mixed.handle, ctypes.c_void_p(hb.data_ptr()),
                                                   ctypes.c_void_p(hx.data_ptr()), None,
                                                   ctypes.byref(st_)))
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = replica_value(world, n_free, opt.steps, e2e_ms)
    x_mixed = x.cpu().numpy()
    x_e2e = hx.numpy().copy()
    mixed_bytes = mixed.device_bytes()
    levels = mixed.levels()
    phases_mixed = setup_phases(mixed)
    del mixed

    # The plain FP64 form on the same workload.
    plain, setup_fp64 = make(fg.FP64)
    ms64, lat64, its64, _, res64, _ = timed(plain, opt.steps, opt.warmup)
    x_fp64 = x.cpu().numpy()
    phases_fp64 = setup_phases(plain)
    ms64 = max_over_ranks(ms64)
    value64 = replica_value(world, n_free, opt.steps, ms64)
    del plain

    cpu = None
    errors = None
    if rank == 0 and world == 1 and not opt.no_cpu_baseline:
        try:
            ref = oracle_solve_rate(A, rhs, facts["oracle_solver"], tol, facts["direct_xyz"])
            cpu = {"value": ref["rate"], "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"1 full solve of the same system by the oracle (reference "
                             f"algorithm: FP64 PCG + the reference's multigrid smoothers), "
                             f"{ref['iterations']} iterations, {ref['solve_s']:.2f} s (setup "
                             f"{ref['setup_s']:.1f} s excluded)",
                   "all_cores": {"value": ref["rate_all"], "cores": ref["cores"],
                                 "sample": "the same solve with the matrix and dot products "
                                           "on all host cores (smoothers sequential)"}}
            # The device solutions of the timed runs (the last step's) against the oracle's.
            errors = {"mixed": error_vs_oracle(x_mixed, ref),
                      "fp64": error_vs_oracle(x_fp64, ref),
                      "e2e": error_vs_oracle(x_e2e, ref),
                      "oracle_residual": {"same_tol": ref["residual"],
                                          "tight": ref["residual_tight"]},
                      # How far the reference's own solution at the same tolerance is from
                      # the converged one: the scale of any two solutions' distance at 1e-8.
                      "oracle_same_tol_vs_1e-12": float(
                          np.linalg.norm(ref["x_tol"] - ref["x_tight"])
                          / np.linalg.norm(ref["x_tight"])),
                      "definition": "|x - x_oracle|_2 / |x_oracle|_2; the oracle's PCG-MG "
                                    "(the reference's algorithm) at the same tolerance, the "
                                    "same continued to 1e-12, and (<= 40,000 unknowns) its "
                                    "multifrontal Cholesky"}
        except Exception as e:  # the baseline is reported, never the product
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"failed: {e}"}

    lat_ms = np.array(lat) * 1e3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": opt.steps,
        "warmup": opt.warmup, "ms_per_step": ms_max / opt.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 outer",
        "data": "synthetic",
        "config": workload_config(facts["text"], n_free, nnz, tol, world),
        "levels": levels,
        "latency_ms": {"p50": float(np.percentile(lat_ms, 50)),
                       "p99": float(np.percentile(lat_ms, 99))},
        "iterations": {"mixed": int(np.median(its)), "fp64": int(np.median(its64))},
        "true_residual": {"mixed": float(max(res)), "fp64": float(max(res64))},
        "fp64": {"value": value64, "unit": UNIT, "ms_per_step": ms64 / opt.steps,
                 "p50_ms": float(np.percentile(np.array(lat64) * 1e3, 50)),
                 "p99_ms": float(np.percentile(np.array(lat64) * 1e3, 99))},
        "mixed_over_fp64": value / value64,
        "setup_s": {"assembly": assemble_s, "submatrix_and_rhs": reduce_s,
                    "solver_mixed": setup_mixed, "solver_fp64": setup_fp64,
                    "phases_mixed": phases_mixed, "phases_fp64": phases_fp64},
        "including_setup": world * n_free / (assemble_s + reduce_s + setup_mixed
                                             + ms_max / opt.steps / 1e3),
        "device_bytes": mixed_bytes,
        "roofline": ({"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                      "frac": achieved / peak, "peak_kind": peak_kind,
                      "kernel": "k_cheb_step<float> (finest level)",
                      "bytes_per_launch": kbytes.value, "launch_ms": kms.value,
                      "traffic": traffic.get("bytes_per_launch") if traffic else None}
                     if roof_ok else
                     {"bound": "latency", "achieved": None, "peak": peak, "unit": "GB/s",
                      "frac": None, "note": "no smoothing level: launch- and latency-bound"}),
        "cpu_baseline": cpu,
        "error_vs_oracle": errors,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n_free,
                "d2h_bytes_per_step": 8 * n_free},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()

# ------------------------------------------------------------------ the batched workload
BATCH_RHS = 16


def batch_members(count, seed=SEED):
    """The batched workload's cantilevers (P1 elasticity, cells log-uniform in 10x1x1 ..
    80x8x8, E uniform in [50, 250] GPa, nu in [0.25, 0.35], 16 random top-face traction load
    cases each), numpy PCG64 ``seed``."""
    from femahoy_b200 import meshgen as mg
    rng = np.random.default_rng(seed)
    return [mg.random_cantilever_p1(rng, nrhs=BATCH_RHS) for _ in range(count)]


def batch_systems(members):
    """Device matrices, grid unknowns and right sides (rows, 16) of the members."""
    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg
    mats, unknowns, rhs = [], [], []
    for p, loads in members:
        K = fg.Csr.assemble(fg.P1_ELASTIC, p.xyz, p.nodes, p.coef)
        mats.append(K.submatrix(p.free))
        rhs.append(np.stack([fg.reduced_rhs(K, loads[r], p.values, p.free)
                             for r in range(BATCH_RHS)], axis=1))
        planes, pts, comp = mg.grid_unknowns(p)
        unknowns.append(fg.Unknowns.Grid(fg.Level(planes, pts, comp)))
    return mats, unknowns, rhs


def oracle_batch_rate(members, rhs, budget_s=20.0):
    """The reference's algorithm on the members, 1 right side at a time (the oracle's PCG with
    the reference's multigrid, FP64, 1 thread), until ``budget_s`` of solving: (DOF-solves/s,
    members, solves, seconds)."""
    import oracle
    from femahoy_b200 import meshgen as mg
    dofs, spent, solves, used = 0, 0.0, 0, 0
    for (p, _), b in zip(members, rhs):
        Ko = oracle.pattern(p.n_unknowns, oracle.dof_elements(p.nodes))
        Ko.assemble(1, p.xyz, p.nodes, p.coef)
        Ao = Ko.submatrix(p.free)
        planes, pts, comp = mg.grid_unknowns(p)
        so = oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
        used += 1
        for r in range(b.shape[1]):
            t0 = time.perf_counter()
            so.solve(b[:, r], tol=TOL)
            spent += time.perf_counter() - t0
            dofs += Ao.n
            solves += 1
            if spent >= budget_s:
                return dofs / spent, used, solves, spent
    return dofs / spent, used, solves, spent


def run_batch(opt, rank, world, local):
    import torch

    import femahoy_b200 as fg
    from femahoy_b200.batch import Batch

    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    lib = fg.lib()
    members = batch_members(opt.systems, SEED + rank)
    t0 = time.perf_counter()
    mats, unknowns, rhs = batch_systems(members)
    assemble_s = time.perf_counter() - t0

    def make(precision):
        t = time.perf_counter()
        bt = Batch(mats, unknowns, BATCH_RHS, precision=precision,
                   options=fg.Options(precision=precision,
                                      smoother=opt.smoother)).with_tol(TOL)
        return bt, time.perf_counter() - t

    def timed(bt, steps, warmup, clocks=None):
        packed = torch.from_numpy(bt.pack(rhs).ravel()).cuda()
        x = torch.zeros_like(packed)
        stream = torch.cuda.ExternalStream(bt.stream())
        for _ in range(warmup):
            with torch.cuda.stream(stream):
                x.zero_()
            bt.solve_device(packed, x)
        barrier()
        stream.synchronize()
        if clocks:
            clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        e0.record(stream)
        for _ in range(steps):
            with torch.cuda.stream(stream):
                x.zero_()
            stats.append(bt.solve_device(packed, x))
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop() if clocks else None
        return e0.elapsed_time(e1), stats, clk

    mixed, setup_mixed = make(fg.MIXED)
    batch_phases = setup_phases(mixed)
    rows = mixed.rows
    clocks = Clocks(torch.cuda.current_device())
    ms, stats, clk = timed(mixed, opt.steps, opt.warmup, clocks)
    ms = max_over_ranks(ms)
    value = world * rows * BATCH_RHS * opt.steps / (ms / 1e3)
    kms, kbytes = mixed.kernel_time(50)
    peak, peak_kind = measured_peak()
    achieved = kbytes / (kms * 1e-3) / 1e9

    # e2e: the host C ABI from pinned host memory, copies inside the timed region.
    hb = torch.from_numpy(mixed.pack(rhs).ravel()).pin_memory()
    hx = torch.zeros_like(hb).pin_memory()
    st_ = fg._lib.BatchStats_t()
    stream = torch.cuda.ExternalStream(mixed.stream())

    def host_solve():
        hx.zero_()
        fg._lib.check(lib.femgpu_batch_solve(mixed.handle, ctypes.c_void_p(hb.data_ptr()),
                                             ctypes.c_void_p(hx.data_ptr()), None,
                                             ctypes.byref(st_)))
    for _ in range(opt.warmup):
        host_solve()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(opt.steps):
        host_solve()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    levels = mixed.levels()
    nbytes = mixed.device_bytes()
    del mixed

    plain, setup_fp64 = make(fg.FP64)
    ms64, stats64, _ = timed(plain, opt.steps, opt.warmup)
    ms64 = max_over_ranks(ms64)
    value64 = world * rows * BATCH_RHS * opt.steps / (ms64 / 1e3)
    del plain

    cpu = None
    if rank == 0 and world == 1 and not opt.no_cpu_baseline:
        rate, used, solves, spent = oracle_batch_rate(members, rhs)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{solves} single-right-side solves of the first {used} members by the "
                         f"oracle (reference algorithm: FP64 PCG + line Gauss-Seidel MG, its "
                         f"coarse direct solve up to 3000 unknowns), {spent:.1f} s, setup "
                         f"excluded"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": opt.steps,
        "warmup": opt.warmup, "ms_per_step": ms / opt.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 outer",
        "data": "synthetic",
        "config": {
            "workload": f"batched: {opt.systems} P1 elasticity cantilevers (cells log-uniform "
                        f"10x1x1..80x8x8, E in [50,250] GPa, nu in [0.25,0.35], seed {SEED}) x "
                        f"{BATCH_RHS} random top-face load cases, 1 batched solve to 1e-8 per "
                        f"step, mixed precision",
            "free_dofs": rows, "pairs": opt.systems * BATCH_RHS, "tol": TOL, "levels": levels,
            "flush": "inputs larger than L2 (operators and 16-column vectors of the batch)",
            "parallelism": f"replicas x{world}",
        },
        "iterations": {"max": int(max(s.max_iterations for s in stats)),
                       "mean": float(np.mean([s.mean_iterations for s in stats])),
                       "fp64_max": int(max(s.max_iterations for s in stats64))},
        "true_residual": {"mixed": float(max(s.max_true_residual for s in stats)),
                          "fp64": float(max(s.max_true_residual for s in stats64))},
        "not_converged": int(sum(s.not_converged for s in stats)),
        "restarts": {"mixed": int(sum(s.restarts for s in stats)),
                     "fp64": int(sum(s.restarts for s in stats64))},
        "latency_ms": {"p50": float(np.percentile([s.seconds * 1e3 for s in stats], 50)),
                       "p99": float(np.percentile([s.seconds * 1e3 for s in stats], 99))},
        "fp64": {"value": value64, "unit": UNIT, "ms_per_step": ms64 / opt.steps},
        "mixed_over_fp64": value / value64,
        "setup_s": {"assembly": assemble_s, "batch_mixed": setup_mixed,
                    "batch_fp64": setup_fp64, "phases_mixed": batch_phases},
        "device_bytes": nbytes,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": "k_bcheb_step3<float,16> (finest level, 3x3 blocks)",
                     "bytes_per_launch": kbytes, "launch_ms": kms, "traffic": None},
        "cpu_baseline": cpu,
        "e2e": {"value": world * rows * BATCH_RHS * opt.steps / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 2 * 8 * rows * BATCH_RHS,
                "d2h_bytes_per_step": 8 * rows * BATCH_RHS},
        "gpu_launches": int(sum(s.launches for s in stats)) + opt.steps,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ continuous batching
STREAM_RATES = (500, 2000, 8000, 32000)
STREAM_REQUESTS = 3000


def run_stream(opt, rank, world, local):
    """Continuous batching: the 256 cantilevers of the batched workload stay resident in 1 batch
    with 16 slots each; a seeded Poisson stream of single load cases (a random member and load
    case each) at each rate of STREAM_RATES is submitted to femgpu_stream_*, whose device loop
    admits each request into a free slot of its member while the others iterate. Reported per
    rate: p50 / p99 latency (submission to the solution on the host), throughput in DOF-solves/s
    over the replay, and the packing (requests served per loop iteration). Each solution is
    checked bit for bit against the batch's own solve of the same load case."""
    import threading

    import torch

    import femahoy_b200 as fg
    from femahoy_b200.batch import Batch, Stream

    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    members = batch_members(opt.systems, SEED + rank)
    mats, unknowns, rhs = batch_systems(members)
    opts = fg.Options(precision=fg.MIXED)
    ref_batch = Batch(mats, unknowns, BATCH_RHS, precision=fg.MIXED, options=opts).with_tol(TOL)
    ref, _ = ref_batch.solve(rhs)
    del ref_batch
    batch = Batch(mats, unknowns, BATCH_RHS, precision=fg.MIXED, options=opts).with_tol(TOL)
    stream = Stream(batch)
    rng = np.random.default_rng(SEED + 7)
    # Warm-up: 1 request per member.
    for t in [stream.submit(k, rhs[k][:, 0]) for k in range(len(members))]:
        stream.wait(t)
    rates = []
    identical = total = 0
    for rate in STREAM_RATES:
        n = STREAM_REQUESTS
        gaps = rng.exponential(1.0 / rate, n)
        picks = [(int(rng.integers(len(members))), int(rng.integers(BATCH_RHS))) for _ in range(n)]
        tickets = [None] * n
        loops0, served0 = stream.counts()

        def submitter():
            t0 = time.perf_counter()
            due = 0.0
            for i, (k, r) in enumerate(picks):
                due += gaps[i]
                while time.perf_counter() - t0 < due:
                    pass
                tickets[i] = stream.submit(k, rhs[k][:, r])

        barrier()
        t_start = time.perf_counter()
        th = threading.Thread(target=submitter)
        th.start()
        lat, dofs = [], 0
        for i, (k, r) in enumerate(picks):
            while tickets[i] is None:
                time.sleep(0)
            x, res = stream.wait(tickets[i])
            lat.append(res.latency_s)
            dofs += len(x)
            total += 1
            identical += int(np.array_equal(x.view(np.uint64), ref[k][:, r].view(np.uint64)))
        th.join()
        wall = time.perf_counter() - t_start
        loops1, served1 = stream.counts()
        lat_ms = np.array(lat) * 1e3
        rates.append({"rate_per_s": rate, "requests": n,
                      "p50_ms": float(np.percentile(lat_ms, 50)),
                      "p99_ms": float(np.percentile(lat_ms, 99)),
                      "throughput": world * dofs / max_over_ranks(wall),
                      "served_per_s": n / wall,
                      "packing": (served1 - served0) / max(1, loops1 - loops0),
                      "loop_iterations": loops1 - loops0})
    stream.close()
    line = {
        "metric": "DOF-solves/s of a Poisson request stream under continuous batching; p50/p99 "
                  "latency",
        "value": rates[-1]["throughput"], "unit": UNIT, "n_gpus": world,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {"workload": f"{opt.systems} resident P1 elasticity cantilevers (the batched "
                               f"workload), 16 slots each; Poisson arrivals of single load "
                               f"cases (seed {SEED}), {STREAM_REQUESTS} requests per rate, to "
                               f"1e-8, mixed precision", "tol": TOL,
                   "parallelism": f"replicas x{world}"},
        "rates": rates,
        "bit_identical_to_batch_solve": f"{identical}/{total}",
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ the serving workload
SERVE_BUDGET = 150 << 30
SERVE_SLOTS = 4


def serve_stream(count, seed=SEED):
    """The request stream: each request names a mesh; 30 % reuse an earlier mesh with a new
    right side, the others bring a new box mesh of log-uniform 10k .. 3M unknowns, half P1 heat
    (lognormal conductivity), a quarter P1 and a quarter P2 elasticity. Returns the requests
    [(mesh id, rhs seed)] and the mesh specs {id: (kind, cells)}."""
    rng = np.random.default_rng(seed)
    meshes, reqs = {}, []
    for i in range(count):
        if meshes and rng.uniform() < 0.3:
            reqs.append((int(rng.choice(list(meshes))), int(rng.integers(1 << 30))))
            continue
        dofs = float(np.exp(rng.uniform(np.log(1e4), np.log(3e6))))
        u = rng.uniform()
        if u < 0.5:
            kind, n = "heat", max(2, int(round(dofs ** (1 / 3))) - 1)
        elif u < 0.75:
            kind, n = "p1", max(2, int(round((dofs / 3) ** (1 / 3))) - 1)
        else:
            kind, n = "p2", max(2, int(round(((dofs / 3) ** (1 / 3) - 1) / 2)))
        mid = len(meshes)
        meshes[mid] = (kind, n)
        reqs.append((mid, int(rng.integers(1 << 30))))
    return reqs, meshes


def serve_mesh(kind, n):
    """The client's model of a mesh spec: the problem (host arrays), and the box for P2."""
    from femahoy_b200 import meshgen as mg
    if kind == "heat":
        return mg.heat_cube(n, seed=SEED + n), None
    if kind == "p1":
        return mg.cantilever_p1(dims=(n, n, n), lengths=(2.5 * n,) * 3), None
    return None, mg.box(n, n, n, (2.5 * n,) * 3)


def serve_setup(kind, prob, box):
    """The server's side of a new mesh: assembly, the free system, its right side and the
    solver (mixed precision, 1e-8). Returns (solver, rhs, free unknowns)."""
    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg
    if kind == "p2":
        q = fg.Quadratic.new(box.points, box.tets)
        prob = mg.beam_p2(q.edges, q.tets, mesh=box)
    code = {"heat": fg.P1_HEAT, "p1": fg.P1_ELASTIC, "p2": fg.P2_ELASTIC}[kind]
    K = fg.Csr.assemble(code, prob.xyz, prob.nodes, prob.coef)
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    del K
    if kind == "p2":
        P, coarse = fg.prolongation(prob.xyz, box.n, q.edges, prob.free)
        u = fg.Unknowns.Quadratic(prob.xyz[prob.free // 3], P, coarse)
    else:
        planes, pts, comp = mg.grid_unknowns(prob)
        u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    s = fg.Solver(A, u, fg.Method.Multigrid, precision=fg.MIXED).with_tol(TOL)
    return s, rhs, A.n


def run_serve(opt, rank, world, local):
    """Replays the request stream at each arrival rate through a fresh server. At its Poisson
    arrival time a request whose mesh is resident goes straight to the server; one that names a
    new mesh waits for 1 of `--builders` builder threads (each builds 1 mesh at a time: assembly
    and hierarchy) that hands the solver to the server and then submits the requests that waited
    for it. A request's
    latency runs from its arrival to the end of its solve (the server's own clock from
    submission to the end of the solve, plus the time before submission)."""
    import queue
    import threading

    import torch

    import femahoy_b200 as fg
    from femahoy_b200.serve import Server

    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    reqs, specs = serve_stream(opt.requests, SEED + rank)
    t0 = time.perf_counter()
    models = {mid: serve_mesh(*spec) for mid, spec in specs.items()}
    client_s = time.perf_counter() - t0
    rates = [float(r) for r in opt.rates.split(",")]
    # Warm-up: 1 small solve of each kind through a server (CUDA context, kernels, graphs).
    warm = Server(slots=1, budget_bytes=SERVE_BUDGET)
    for kind in ("heat", "p1", "p2"):
        prob, box = serve_mesh(kind, 6)
        sv, rhs, _ = serve_setup(kind, prob, box)
        warm.put(0, sv)
        warm.wait(warm.submit(0, rhs))
    del warm
    barrier()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    sweep = []
    launches = 0
    for rate in rates:
        server = Server(slots=SERVE_SLOTS, budget_bytes=SERVE_BUDGET)
        lock = threading.Lock()
        ready = {}     # mesh id -> (rhs, free unknowns) once its solver is resident
        pending = {}   # mesh id -> requests that arrived before its solver was ready
        submitted = []  # (request index, mesh id, arrival, submit time, ticket, resident)
        builds = queue.Queue()
        rng = np.random.default_rng(SEED + int(rate))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))

        def submit(i, mid, resident):
            rhs, n = ready[mid]
            r = np.random.default_rng(reqs[i][1])
            b = rhs * r.uniform(0.5, 2.0) + 0.2 * np.abs(rhs).max() * r.standard_normal(n)
            t = time.perf_counter()
            submitted.append((i, mid, t, server.submit(mid, b), resident))

        def builder():
            # 1 build at a time per thread: assembly and hierarchy of a new mesh, then the
            # requests that waited for it go to the server.
            while True:
                mid = builds.get()
                if mid is None:
                    return
                sv, rhs, n = serve_setup(specs[mid][0], *models[mid])
                server.put(mid, sv)
                with lock:
                    ready[mid] = (rhs, n)
                    for i in pending.pop(mid):
                        submit(i, mid, False)

        workers = [threading.Thread(target=builder) for _ in range(opt.builders)]
        for w in workers:
            w.start()
        start = time.perf_counter()
        for i, (mid, _) in enumerate(reqs):
            wait = start + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            with lock:
                if mid in ready:
                    submit(i, mid, True)
                elif mid in pending:
                    pending[mid].append(i)
                else:
                    pending[mid] = [i]
                    builds.put(mid)
        for _ in workers:
            builds.put(None)
        for w in workers:
            w.join()
        records = []
        for i, mid, t_sub, ticket, resident in sorted(submitted):
            x, st, solve_s = server.wait(ticket)
            end = t_sub + solve_s
            records.append({"n": ready[mid][1], "hit": resident,
                            "latency": end - (start + arrivals[i]), "end": end,
                            "iterations": st.iterations, "true_residual": st.true_residual,
                            "launches": st.launches, "kind": specs[mid][0]})
        span = max(r["end"] for r in records) - (start + arrivals[0])
        lat = np.array([r["latency"] for r in records]) * 1e3
        hits = np.array([r["latency"] for r in records if r["hit"]]) * 1e3
        launches += sum(r["launches"] for r in records)
        sweep.append({
            "rate_per_s": rate, "requests": len(records),
            "throughput": sum(r["n"] for r in records) / span,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "resident_p50_ms": float(np.percentile(hits, 50)) if len(hits) else None,
            "resident_p99_ms": float(np.percentile(hits, 99)) if len(hits) else None,
            "max_true_residual": float(max(r["true_residual"] for r in records)),
            "resident_bytes": server.resident_bytes, "span_s": span})
        del server
    clk = clocks.stop()
    top = sweep[-1]
    # The slowest replica sets the whole-job figure.
    value = -max_over_ranks(-top["throughput"])
    line = {
        "metric": METRIC, "value": world * value, "unit": UNIT, "n_gpus": world,
        "steps": len(reqs), "warmup": 3, "ms_per_step": top["span_s"] * 1e3 / len(reqs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {
            "workload": f"serving: {len(reqs)} Poisson-arriving solve requests per rate "
                        f"(seed {SEED}), box meshes of log-uniform 10k..3M unknowns (1/2 P1 "
                        f"heat, 1/4 P1, 1/4 P2 elasticity), 30 % reuse a resident mesh with a "
                        f"new right side; setup of a new mesh (assembly, hierarchy) counts in "
                        f"its request's latency; {SERVE_SLOTS} slots, 150 GB budget, 1e-8",
            "meshes": len(specs), "rates": rates, "tol": TOL,
            "parallelism": f"replicas x{world}"},
        "sweep": sweep,
        "latency_ms": {"p50": top["p50_ms"], "p99": top["p99_ms"]},
        "client_mesh_generation_s": client_s,
        "roofline": None,
        "cpu_baseline": None,
        "e2e": {"value": world * value, "unit": UNIT,
                "note": "the stream runs through the host API: every value is end to end"},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _plumbing(world, backend="nccl"):
    """The process group (N > 1), a barrier that also synchronizes the device, and the max over
    ranks of a number. The path does not shard: the N ranks are independent replicas, and these
    are the only collectives (gloo runs the same steps on the host, for the CPU tests)."""
    import torch
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    on_gpu = backend == "nccl"

    def barrier():
        if world > 1:
            dist.barrier()
        if on_gpu:
            torch.cuda.synchronize()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda" if on_gpu else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return dist, barrier, max_over_ranks


def replica_value(world, units, steps, ms_max):
    """The whole-job figure of N replicas: all ranks' units over the slowest rank's time."""
    return world * units * steps / (ms_max / 1e3)


# ------------------------------------------------------------------ the transient workload
TRANSIENT_METRIC = "DOF-steps/s of backward-Euler transient heat (1 resident operator)"


def run_transient(opt, rank, world, local):
    """The transient loop of heat.rs:686-733 on the 128^3 heat cube: lumped capacity 1 per unit
    volume, dt = 1e-3, from T = 0 with the fixed temperatures of the steady problem; a step is 1
    time step (right side, 1 warm-started solve to 1e-8, the temperatures), mixed form. The
    call is the public host API (load and temperatures in, the last temperatures and 1 frame
    per 10 steps out), so value and e2e are the same measurement; the device time of the solves
    is reported beside it. The CPU baseline runs the oracle's loop for 2 steps."""
    import torch
    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg
    from femahoy_b200.transient import Transient
    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    h = build_problem(opt.cells)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    cap = mg.lumped_capacity(h.mesh, capacity=1.0)
    planes, pts, comp = mg.grid_unknowns(h)
    u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    dt = 1e-3
    t0 = time.perf_counter()
    tr = Transient(K, cap, dt, h.free, u, fg.Method.Multigrid,
                   options=fg.Options(precision=fg.MIXED))
    tr.solver.with_tol(TOL)
    setup_s = time.perf_counter() - t0
    every = 10
    tr.run(opt.warmup, h.load, h.values, output_every=every)
    barrier()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    t0 = time.perf_counter()
    frames, energies, t, st = tr.run(opt.steps, h.load, h.values, output_every=every)
    torch.cuda.synchronize()
    wall = max_over_ranks(time.perf_counter() - t0)
    clk = clocks.stop()
    n_free = tr.nfree
    value = world * n_free * opt.steps / wall
    cpu = None
    if rank == 0 and world == 1 and not opt.no_cpu_baseline:
        import oracle
        k = oracle.pattern(h.n_points, h.nodes)
        k.assemble(0, h.xyz, h.nodes, h.coef)
        t1 = time.perf_counter()
        of, oe, its = oracle.transient(
            k, cap, dt, h.free, h.load, h.values, 2,
            lambda a: oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp,
                                    method="multigrid"), tol=TOL)
        cpu_s = time.perf_counter() - t1
        cpu = {"value": n_free * 2 / cpu_s, "unit": "DOF-steps/s", "cores": 1, "kind": "port",
               "sample": f"the oracle's loop (the reference's algorithm, FP64 PCG + line "
                         f"Gauss-Seidel multigrid) for 2 steps, {its} PCG iterations, "
                         f"{cpu_s:.1f} s including its hierarchy setup"}
    imb = max(abs(e.stored - h.load.sum() - e.fixed) / e.gross for e in energies)
    line = {
        "metric": TRANSIENT_METRIC, "value": value, "unit": "DOF-steps/s", "n_gpus": world,
        "steps": opt.steps, "warmup": opt.warmup, "ms_per_step": 1e3 * wall / opt.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {"workload": f"transient P1 heat, {opt.cells}^3 Kuhn box, lognormal k (seed "
                               f"{SEED}), lumped capacity 1, dt 1e-3, from T = 0, each step "
                               f"solved to 1e-8 from the last temperatures",
                   "free_dofs": n_free, "flush": "inputs larger than L2",
                   "parallelism": f"replicas x{world}"},
        "pcg_iterations_per_step": st.iterations / opt.steps,
        "device_solve_ms_per_step": 1e3 * st.seconds / opt.steps,
        "energy_imbalance": imb, "setup_s": setup_s,
        "roofline": {"bound": "hbm", "achieved": None, "peak": measured_peak()[0],
                     "unit": "GB/s", "frac": None,
                     "note": "the per-step solve is the heat solve of the default line"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "DOF-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8 * h.n_points // every},
        "gpu_launches": st.launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ the modes workload
MODES_METRIC = "modes analyses/s (10 lowest modes, shift-invert subspace iteration)"


def run_modes(opt, rank, world, local):
    """The 10 lowest modes of the 100x10x10 P2 beam (200x20x20 mm, aluminium: E 70 GPa, nu 0.33,
    density 2.7e-9 t/mm^3, clamped at x = 0): K and M assembled on the device, K - shift M solved
    by p-multigrid PCG (mixed) 20 times per subspace iteration (p = 20). A step is 1 whole
    analysis. The CPU baseline solves 1 system of the oracle (the reference's p-multigrid PCG) and
    scales it by the device analysis's solve count, an estimate that leaves out the oracle's
    projections."""
    import torch
    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg
    from femahoy_b200.modes import modes
    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    hexes = opt.workload == "hexmodes"
    cells = None
    t0 = time.perf_counter()
    if hexes:
        # modes.rs:355-420: a box-cell cantilever of steel, the coarse matrices from the cells
        # of K - shift M.
        prob = mg.hex_cantilever(nx=128, ny=16, nz=16, length=8.0, width=1.0, depth=1.0,
                                 e=210e3, nu=0.3, load=0.0)
        free = prob.free
        density = np.full(len(prob.nodes), 7.85e-9)
        Kf = fg.Csr.assemble(fg.HEX8_ELASTIC, prob.xyz, prob.nodes, prob.coef).submatrix(free)
        Mf = fg.Csr.assemble(fg.HEX8_MASS, prob.xyz, prob.nodes, density).submatrix(free)
        origin, cls, keys = mg.hex_classes(prob)
        cells = fg.Cells(origin, cls, fg.hex_elements(keys),
                         fg.hex_mass(keys[:, :3], np.full(len(keys), 7.85e-9)))
        planes, pts, comp = mg.grid_unknowns(prob)
        u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    else:
        box = mg.box(100, 10, 10, (200.0, 20.0, 20.0))
        q = fg.Quadratic.new(box.points, box.tets)
        prob = mg.beam_p2(q.edges, q.tets, mesh=box, seed=SEED)
        density = np.full(len(q.tets), 2.7e-9)
        free = prob.free
        Kf = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, prob.nodes, prob.coef).submatrix(free)
        Mf = fg.Csr.assemble(fg.P2_MASS, prob.xyz, prob.nodes, density).submatrix(free)
        P, coarse = fg.prolongation(prob.xyz, box.n, q.edges, free)
        u = fg.Unknowns.Quadratic(prob.xyz[free // 3], P, coarse)
    assemble_s = time.perf_counter() - t0
    opts = fg.Options(precision=fg.MIXED)
    for _ in range(max(1, opt.warmup)):
        values, _, st = modes(Kf, Mf, 10, u, fg.Method.Multigrid, options=opts, vectors=False,
                              cells=cells)
    barrier()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(opt.steps):
        values, _, st = modes(Kf, Mf, 10, u, fg.Method.Multigrid, options=opts, vectors=False,
                              cells=cells)
    torch.cuda.synchronize()
    wall = max_over_ranks(time.perf_counter() - t0)
    clk = clocks.stop()
    value = world * opt.steps / wall
    cpu = None
    if rank == 0 and world == 1 and not opt.no_cpu_baseline:
        import oracle
        Ko = oracle.Csr.from_arrays(Kf.n, *Kf.arrays())
        Mo = oracle.Csr.from_arrays(Mf.n, *Mf.arrays())
        ptr, idx, val = Ko.arrays()
        Ao = oracle.Csr.from_arrays(Ko.n, ptr, idx, val - st.shift * Mo.arrays()[2])
        if hexes:
            oc = (cells.origin, cells.cls, cells.matrices - st.shift * cells.mass)
            so = oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp,
                               method="multigrid", cells=oc)
        else:
            Po = oracle.Rect.from_arrays(P.rows, P.cols, P.ptr, P.idx, P.val)
            so = oracle.Solver(Ao, "quadratic", xyz=prob.xyz[free // 3], p=Po, coarse=coarse,
                               method="multigrid")
        y = Mo.mul(np.random.default_rng(1).standard_normal(Ko.n))
        t1 = time.perf_counter()
        _, its, _ = so.solve(y, tol=1e-10)
        one = time.perf_counter() - t1
        cpu = {"value": 1.0 / (one * st.solves), "unit": "analyses/s", "cores": 1,
               "kind": "port",
               "sample": f"1 solve of K - shift M by the oracle (the reference's "
                         f"{'cell-based multigrid' if hexes else 'p-multigrid'} PCG, "
                         f"{its} iterations, {one:.1f} s) times the device analysis's "
                         f"{st.solves} solves"}
    line = {
        "metric": MODES_METRIC, "value": value, "unit": "analyses/s", "n_gpus": world,
        "steps": opt.steps, "warmup": opt.warmup, "ms_per_step": 1e3 * wall / opt.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {"workload": (f"10 lowest modes of the 128x16x16 box-cell cantilever of steel "
                                f"({Kf.n} free unknowns), clamped at x = 0, coarse matrices "
                                f"from the cells of K - shift M" if hexes else
                                "10 lowest modes of the 100x10x10 P2 beam (60,000 10-node "
                                f"tets, {Kf.n} free unknowns), clamped at x = 0"),
                   "free_dofs": Kf.n, "subspace_vectors": 20,
                   "flush": "inputs larger than L2", "parallelism": f"replicas x{world}"},
        "eigenvalues": [float(v) for v in values],
        "subspace_iterations": st.iterations, "solves": st.solves,
        "pcg_iterations": st.pcg_iterations, "solve_seconds": st.seconds,
        "assembly_s": assemble_s,
        "roofline": {"bound": "hbm", "achieved": None, "peak": measured_peak()[0],
                     "unit": "GB/s", "frac": None,
                     "note": ("the solves are the cell-based multigrid PCG of K - shift M"
                              if hexes else
                              "the solves are the p-multigrid PCG of the p2beam line")},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "analyses/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 80},
        "gpu_launches": None,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ the recovery workload
RECOVER_METRIC = "recovered points/s (strain, stress, von Mises, principal, peaks)"


def run_recover(opt, rank, world, local):
    """The post-solve recovery of the 200x20x20 P2 beam (elastic_tet.rs:367-427, 482-483): the
    beam solved once (mixed, 1e-8), then a step is 1 recovery of all 674,081 points from the
    resident displacement: mean strain and stress, von Mises and principal stresses, and the
    peaks of 4 parts (cells split by x) with the edges of the clamped face singular. e2e is the
    same through the host C ABI (u from host memory, the results back)."""
    import torch
    import femahoy_b200 as fg
    from femahoy_b200 import meshgen as mg
    from femahoy_b200.recover import Recovery
    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    hexes = opt.workload == "hexrecover"
    if hexes:
        # elastic.rs:615-660: the box grid's recovery after the box-cell cantilever's solve.
        prob = mg.hex_cantilever(nx=256, ny=32, nz=32, length=8.0, width=1.0, depth=1.0,
                                 e=1000.0, nu=0.3, load=-1.0, seed=SEED)
        K = fg.Csr.assemble(fg.HEX8_ELASTIC, prob.xyz, prob.nodes, prob.coef)
        planes, pts, comp = mg.grid_unknowns(prob)
        unknowns = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
        width = 1.0
    else:
        box = mg.box(200, 20, 20, (200.0, 20.0, 20.0))
        q = fg.Quadratic.new(box.points, box.tets)
        prob = mg.beam_p2(q.edges, q.tets, mesh=box, seed=SEED)
        K = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, prob.nodes, prob.coef)
        width = 20.0
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    del K
    if not hexes:
        P, coarse = fg.prolongation(prob.xyz, box.n, q.edges, prob.free)
        unknowns = fg.Unknowns.Quadratic(prob.xyz[prob.free // 3], P, coarse)
    solver = fg.Solver(A, unknowns, fg.Method.Multigrid,
                       options=fg.Options(precision=fg.MIXED)).with_tol(TOL)
    x = np.zeros(A.n)
    solver.solve(rhs, x)
    del solver
    u = prob.values.copy()
    u[prob.free] = x
    xyz, t10 = prob.xyz, prob.nodes
    n, ne = len(xyz), len(t10)
    nparts = 4
    part = (4 * np.arange(ne) // ne).astype(np.uint32)
    on = lambda d, v: xyz[:, d] == v
    singular = (on(0, 0.0) & (on(1, 0.0) | on(1, width) | on(2, 0.0) | on(2, width))).astype(
        np.uint8)
    t0 = time.perf_counter()
    rec = Recovery(xyz, t10, prob.coef, part=part, nparts=nparts, singular=singular, hex=hexes)
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(fg.lib().femgpu_recovery_stream(rec.handle))
    dev = torch.device("cuda", local)
    ud = torch.from_numpy(u).to(dev)
    st = torch.empty((n, 6), dtype=torch.float64, device=dev)
    sn, mi, pr = torch.empty_like(st), torch.empty(n, dtype=torch.float64, device=dev), \
        torch.empty((n, 3), dtype=torch.float64, device=dev)

    def step():
        return rec.run_device(ud, st, sn, mises=mi, principal=pr)

    for _ in range(opt.warmup):
        step()
    barrier()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kms = []
    e0.record(stream)
    for _ in range(opt.steps):
        step()
        kms.append(rec.last_time())
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * n * opt.steps / (ms / 1e3)
    # The recovery kernels alone (CUDA events around them on the recovery stream).
    kernel_ms = float(np.median([k for k, _ in kms]))
    kbytes = kms[-1][1]
    peak, peak_kind = measured_peak()
    achieved = kbytes / (kernel_ms * 1e-3) / 1e9
    # e2e: the host form, u from pinned host memory and all results back to it.
    hu = torch.from_numpy(u).pin_memory().numpy()
    for _ in range(opt.warmup):
        rec.run(hu)
    barrier()
    t0 = time.perf_counter()
    for _ in range(opt.steps):
        out = rec.run(hu)
    e2e_s = time.perf_counter() - t0
    e2e_value = world * n * opt.steps / e2e_s
    cpu = None
    if rank == 0 and world == 1 and not opt.no_cpu_baseline:
        import oracle
        t0 = time.perf_counter()
        ref = oracle.recover(xyz, t10, prob.coef, u, part=part, nparts=nparts,
                             singular=singular, hex=hexes)
        cpu_s = time.perf_counter() - t0
        same = all(np.array_equal(out[k].view(np.uint64), ref[k].view(np.uint64))
                   for k in ("stress", "strain", "mises"))
        cpu = {"value": n / cpu_s, "unit": "points/s", "cores": 1, "kind": "port",
               "sample": f"1 full recovery of the same model by the oracle ({cpu_s:.2f} s); "
                         f"bits identical with the GPU's: {same}"}
    line = {
        "metric": RECOVER_METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": opt.steps, "warmup": opt.warmup, "ms_per_step": ms / opt.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": (f"stress recovery of the 256x32x32 box-cell cantilever "
                                f"({ne} cells with incompatible modes, {n} points, 2 "
                                f"materials) after its solve to 1e-8; 4 parts, clamped-face "
                                f"edges singular" if hexes else
                                f"stress recovery of the 200x20x20 P2 beam (480,000 10-node "
                                f"tets, {n} points) after its solve to 1e-8; 4 parts, "
                                f"clamped-face edges singular"),
                   "points": n, "cells": ne, "flush": "inputs larger than L2",
                   "parallelism": f"replicas x{world}"},
        "setup_s": setup_s,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": ("k_pad_u + k_hex_amplitudes + k_recover_hex_points<peaks> + "
                                "k_peak_final" if hexes else
                                "k_pad_u + k_recover_points<peaks> + k_peak_final"),
                     "bytes_per_launch": kbytes, "launch_ms": kernel_ms, "traffic": None},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": (6 + 6 + 1 + 3) * 8 * n},
        "gpu_launches": (4 if hexes else 3) * opt.steps,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ the direct workload
DIRECT_METRIC = "DOF-solves/s of the direct method (sparse multifrontal factor on the device)"


def run_direct(opt, rank, world, local):
    """The direct method of solve.rs:92-250 above 4,096 unknowns (the reference's choice for P2
    models up to 30,000 unknowns, elastic_tet.rs:52-56): the 50 x 5 x 5 P2 beam (36,300 free
    unknowns), factored once on the device (cholesky.rs:44-167's multifrontal factor in the
    order of order.rs); a step is 1 solve of a resident right side (the 2 triangular solves).
    The solution is checked against the oracle's factor (CPU) and timed beside it."""
    import torch
    import femahoy_b200 as fg
    import oracle
    from femahoy_b200 import meshgen as mg
    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    dims, lengths = (50, 5, 5), (250.0, 25.0, 25.0)
    m = mg.box(*dims, lengths)
    q = fg.Quadratic.new(m.points, m.tets)
    prob = mg.beam_p2(q.edges, q.tets, dims=dims, lengths=lengths, mesh=m, seed=SEED)
    K = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, prob.nodes, prob.coef)
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    xyz = prob.xyz[prob.free // 3]
    P, coarse = fg.prolongation(prob.xyz, m.n, q.edges, prob.free)
    t = time.perf_counter()
    s = fg.Solver(A, fg.Unknowns.Quadratic(xyz, P, coarse), fg.Method.Direct)
    setup_s = time.perf_counter() - t
    b = torch.from_numpy(rhs).cuda()
    x = torch.zeros_like(b)
    for _ in range(opt.warmup):
        s.solve_device(b.data_ptr(), x.data_ptr())
    barrier()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    secs, res, launches = [], [], 0
    for _ in range(opt.steps):
        st = s.solve_device(b.data_ptr(), x.data_ptr())
        secs.append(st.seconds)
        res.append(st.true_residual)
        launches += st.launches
    clk = clocks.stop()
    ms = max_over_ranks(1e3 * sum(secs))
    xh = np.zeros(A.n)
    t0 = time.perf_counter()
    for _ in range(opt.steps):
        s.solve(rhs, xh)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    cpu = None
    err = None
    if rank == 0 and not opt.no_cpu_baseline:
        Ko = oracle.pattern(prob.n_unknowns, oracle.dof_elements(prob.nodes))
        Ko.assemble(2, prob.xyz, prob.nodes, prob.coef)
        t0 = time.perf_counter()
        xd, _ = oracle.direct_solve(Ko.submatrix(prob.free), xyz, rhs)
        cpu_s = time.perf_counter() - t0
        err = float(np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd))
        cpu = {"value": A.n / cpu_s, "unit": "DOF-solves/s", "cores": 1, "kind": "port",
               "sample": "1 factor and solve of the same system by the oracle (its whole direct "
                         "solve, the factor included)"}
    line = {
        "metric": DIRECT_METRIC, "value": replica_value(world, A.n, opt.steps, ms),
        "unit": UNIT, "n_gpus": world, "steps": opt.steps, "warmup": opt.warmup,
        "ms_per_step": ms / opt.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "the direct method on the 50x5x5 P2 beam (36,300 free unknowns)",
                   "free_dofs": A.n, "parallelism": f"replicas x{world}",
                   "flush": "none: each solve reads the factor's L entries (0.11 GB) and its "
                            "block inverses, about the size of L2"},
        "setup_s": setup_s, "true_residual": max(res), "error_vs_oracle": err,
        "describe": s.describe().strip().splitlines()[-1],
        "cpu_baseline": cpu, "roofline": None,
        "e2e": {"value": replica_value(world, A.n, opt.steps, e2e_s * 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * A.n, "d2h_bytes_per_step": 8 * A.n},
        "gpu_launches": launches, "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ the prism-mesh workload
PRISM_METRIC = "DOF-solves/s at 1e-8 rel. residual of P2 elasticity on the reference's prism mesh"


def run_prism(opt, rank, world, local):
    """elastic_tet.rs:88-337's path end to end on the reference's own mesh (prism.rs:170): a
    4 x 2 x 0.25 plate with 3 round holes and a boss of a second material on top, meshed
    (footprint triangulation on the host, extrusion on the device), Quadratic, P2 assembly,
    clamped at x = 0 with a downward load at x = 4, p-multigrid to the corners and z-only
    geometric levels (the points lie on the planes of the axis). The stage seconds are reported;
    a step is 1 mixed solve from x = 0 to 1e-8; e2e is the same through the host C ABI."""
    import torch
    import femahoy_b200 as fg
    from femahoy_b200 import prism as P
    torch.cuda.set_device(local)
    dist, barrier, max_over_ranks = _plumbing(world)
    lib = fg.lib()
    stages = {}
    t = time.perf_counter()
    hole = lambda c, r: P.Outline.circle(c, r)  # noqa: E731
    plate = P.Part("plate", 0, 0, (0.0, 0.0, 0.0), (0.0, 0.0, 0.25),
                   P.Footprint(P.Outline.polygon([(0, 0), (4, 0), (4, 2), (0, 2)]),
                               [hole((1.0, 1.0), 0.3), hole((2.2, 0.6), 0.2),
                                hole((3.2, 1.3), 0.25)]))
    boss = P.Part("boss", 1, 1, (0.0, 0.0, 0.25), (0.0, 0.0, 0.45),
                  P.Footprint(P.Outline.polygon([(1.8, 1.1), (2.8, 1.1), (2.8, 1.8),
                                                 (1.8, 1.8)]), []))
    tm = P.mesh([plate, boss], 2, P.Spacing(opt.prism_cell, 1.3, 2), 250_000,
                "the mesh has more points than the solver takes")
    stages["mesh (2D on the host, extrusion on the device)"] = time.perf_counter() - t
    t = time.perf_counter()
    q = fg.Quadratic.new(tm.points, tm.tets)
    stages["quadratic"] = time.perf_counter() - t
    n = len(q.points)
    e = np.array([200e9, 70e9])[tm.part]
    nu = np.array([0.3, 0.33])[tm.part]
    coef = np.stack([e, nu], axis=1)
    t = time.perf_counter()
    K = fg.Csr.assemble(fg.P2_ELASTIC, q.points, q.tets, coef)
    stages["assembly"] = time.perf_counter() - t
    fixed = np.repeat(q.points[:, 0] == 0.0, 3)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    load = np.zeros(3 * n)
    at = np.nonzero(q.points[:, 0] == 4.0)[0]
    load[3 * at + 2] = -1e3 / len(at)
    t = time.perf_counter()
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, load, np.zeros(3 * n), free)
    Pm, coarse = fg.prolongation(q.points, len(tm.points), q.edges, free)
    stages["submatrix, right side, prolongation"] = time.perf_counter() - t
    t = time.perf_counter()
    s = fg.Solver(A, fg.Unknowns.Quadratic(q.points[free // 3], Pm, coarse),
                  fg.Method.Multigrid,
                  options=fg.Options(precision=fg.MIXED, axes=4)).with_tol(TOL)
    stages["solver"] = time.perf_counter() - t
    b = torch.from_numpy(rhs).cuda()
    x = torch.zeros_like(b)
    stream = torch.cuda.ExternalStream(lib.femgpu_solver_stream(s.handle))
    if opt.breakdown:
        for _ in range(3):
            with torch.cuda.stream(stream):
                x.zero_()
            st = s.solve_device(b.data_ptr(), x.data_ptr())
        if rank == 0:
            print(f"== mixed: {st.iterations} iterations, {st.seconds * 1e3:.3f} ms per solve")
            print(s.describe())
            print(s.breakdown(), flush=True)
        return
    for _ in range(opt.warmup):
        with torch.cuda.stream(stream):
            x.zero_()
        s.solve_device(b.data_ptr(), x.data_ptr())
    barrier()
    stream.synchronize()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    its, res, launches = [], [], 0
    e0.record(stream)
    for _ in range(opt.steps):
        with torch.cuda.stream(stream):
            x.zero_()
        st = s.solve_device(b.data_ptr(), x.data_ptr())
        its.append(st.iterations)
        res.append(st.true_residual)
        launches += st.launches + 1
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    barrier()
    xh = np.zeros(A.n)
    t0 = time.perf_counter()
    for _ in range(opt.steps):
        s.solve_zero(rhs, xh)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    kms, kbytes = ctypes.c_double(), ctypes.c_double()
    roof = None
    if lib.femgpu_solver_kernel_time(s.handle, 0, 50, ctypes.byref(kms), ctypes.byref(kbytes)) == 0:
        peak, kind = measured_peak()
        ach = kbytes.value / (kms.value / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_kind": kind, "kernel": "the finest FP32 smoothing step",
                "bytes_per_launch": kbytes.value, "launch_ms": kms.value, "traffic": None}
    line = {
        "metric": PRISM_METRIC, "value": replica_value(world, A.n, opt.steps, ms),
        "unit": UNIT, "n_gpus": world, "steps": opt.steps, "warmup": opt.warmup,
        "ms_per_step": ms / opt.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {"workload": f"P2 elasticity of a plate with 3 holes and a boss, prism mesh "
                               f"max_cell {opt.prism_cell} ({len(tm.points)} points, "
                               f"{len(tm.tets)} tetrahedra, {tm.triangles} triangles x "
                               f"{tm.planes} planes)", "free_dofs": A.n, "tol": TOL,
                   "levels": s.levels(), "flush": "inputs larger than L2",
                   "parallelism": f"replicas x{world}"},
        "iterations": {"max": max(its)}, "true_residual": max(res),
        "stages_s": stages, "roofline": roof, "cpu_baseline": None,
        "e2e": {"value": replica_value(world, A.n, opt.steps, e2e_s * 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * A.n, "d2h_bytes_per_step": 8 * A.n},
        "gpu_launches": launches, "clocks": clk,
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
    if opt.workload in ("recover", "hexrecover"):
        run_recover(opt, rank, world, local)
    elif opt.workload == "transient":
        run_transient(opt, rank, world, local)
    elif opt.workload in ("modes", "hexmodes"):
        run_modes(opt, rank, world, local)
    elif opt.workload == "batch":
        run_batch(opt, rank, world, local)
    elif opt.workload == "serve":
        run_serve(opt, rank, world, local)
    elif opt.workload == "stream":
        run_stream(opt, rank, world, local)
    elif opt.workload == "prism":
        run_prism(opt, rank, world, local)
    elif opt.workload == "direct":
        run_direct(opt, rank, world, local)
    else:
        run_ours(opt, rank, world, local)


if __name__ == "__main__":
    main()
