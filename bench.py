"""Benchmark: assembled+solved DoF/s at relative residual 1e-10.

Workloads (--workload; all inputs seeded and synthetic):

* c2 (default): P2 tetrahedral Poisson, 48^3 x 6 jittered Kuhn box (663,552
  cells, 912,673 DoFs), lognormal cell coefficient, sin*sin*sin source at the
  4-point rule, homogeneous Dirichlet.
* c1: P1 Poisson on unit_square_mesh(65) (8192 triangles, 4225 nodes), f = 1.
* c3 --order k: first-kind Nedelec curl mu^-1 curl + I on the 24^3 x 6 Kuhn
  box, mu^-1 = 1 / 1000 / 1 in three slabs along z, J = (0, 0, 1) in the
  central slab, zero tangential trace; --assembly tf32x3 contracts the
  element matrices of orders 3-6 on the tensor cores (c5 too).
* c5: Nedelec order 6 on the 12^3 x 6 box jittered +-0.05h, mu^-1 ~ U[0.5, 2],
  kappa = 10, smooth random trig source.

One step = assemble (geometry + contraction + scatter + load + constrained
reduction) + mixed-precision Jacobi-PCG until the true FP64 residual
||b - A x|| / ||b|| <= 1e-10 (or, where FP64 cannot represent a solution
that good, until the true residual stops falling; the line then reports the
residual reached and the FP64 rounding floor eps || |A| |x| || / ||b||), from
inputs resident in HBM.  The topology (DoF numbering, CSC pattern, slot maps)
is built once per mesh and reported as setup.  `e2e` repeats the step
through the public host-array API with the host<->device copies inside the
timed region.  With --gpus N > 1 every rank solves its own replica (the path
has no exchange step for independent systems); value = total DoFs solved /
max over ranks of the time.

`--impl reference` times the FP64 CPU restatement of the reference path
(oracle/) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("assembled+solved DoF/s at rel. residual 1e-10 (mixed vs FP64); "
          "p50/p99 solve latency")
TOL = 1e-10
EPS = float(np.finfo(np.float64).eps)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one pcg_kernel
# launch on the 48^3 P2 workload, from an ncu capture of
# `bench.py --steps 1 --warmup 3 --no-cpu --no-e2e --no-fp64 --serving-requests 0`, and the
# algorithmic bytes of that launch; the live launch's traffic is scaled by
# its own algorithmic bytes.
PCG_TRAFFIC_BYTES = 101.803065e9 + 3.318534e9
PCG_TRAFFIC_ALG_BYTES = 159007138196.0


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c5"])
    ap.add_argument("--order", type=int, default=1, help="Nedelec order of the c3 workload")
    ap.add_argument("--size", type=int, default=0, help="mesh size (0: the workload's own)")
    ap.add_argument("--assembly", default="fp64", choices=["fp64", "tf32x3"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "mixed16"],
                    help="inner SpMV operator of the mixed solve: FP32 or row-scaled FP16")
    ap.add_argument("--autotune", action="store_true", help="autotune launch shapes in setup")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=-1,
                    help="requests of the serving leg (0 skips it; default 1024 for c2; the "
                         "full C4 stream is 4096)")
    ap.add_argument("--serving-rate", type=float, default=15.0)
    ap.add_argument("--max-iterations", type=int, default=1000000)
    ap.add_argument("--timeout", type=float, default=60.0, help="device time limit of one solve")
    ap.add_argument("--ref-iterations", type=int, default=0,
                    help="reference arm of c3 orders >= 2 and c5: the FP64 Jacobi-PCG iteration "
                         "count to scale the sampled iterations to (a full CPU solve takes hours)")
    a = ap.parse_args(argv)
    if a.serving_requests < 0:
        a.serving_requests = 1024 if a.workload == "c2" else 0
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


# ---------------------------------------------------------------- workloads

class Workload:
    """One measured configuration: its mesh, coefficients and source, how the
    GPU problem is created, and the oracle's restatement of the reference
    pipeline on the same inputs."""

    def __init__(self, args, mesh=None):
        from fortfem_b200 import synth
        from fortfem_b200._capi import (FFG_RULE_DEGREE_TWO, FFG_RULE_DUFFY, FFG_TETRA_LAGRANGE,
                                        FFG_TETRA_NEDELEC, FFG_TRIANGLE_P1)
        self.kind = args.workload
        self.rule, self.qdeg = FFG_RULE_DUFFY, 0
        self.cell_b = None
        if self.kind == "c2":
            n = args.size or 48
            c = synth.p2_poisson_case(n, mesh=mesh)
            self.family, self.degree = FFG_TETRA_LAGRANGE, 2
            self.rule = FFG_RULE_DEGREE_TWO
            self.v, self.t, self.cell_a = c.vertices, c.cells, c.cell_coefficient
            self.coef_a, self.coef_b = 1.0, 0.0
            self._src = lambda p: c.source(p[..., 0], p[..., 1], p[..., 2])
            self.name = f"p2_tetra_poisson_{n}cube_x6_jittered_lognormal"
            self.desc = dict(degree=2, quadrature="4-point degree-two rule")
        elif self.kind == "c1":
            n = args.size or 65
            if mesh is None:
                from fortfem_b200 import api
                v, t = api.unit_square_mesh(n)
            else:
                v, t = mesh(n)
            self.family, self.degree = FFG_TRIANGLE_P1, 1
            self.v, self.t, self.cell_a = v, t, None
            self.coef_a, self.coef_b = 1.0, 0.0
            self._src = lambda p: np.ones(p.shape[:-1])
            self.name = f"p1_poisson_unit_square_{n}"
            self.desc = dict(degree=1, quadrature="closed-form P1 (3-point equivalent)")
        else:
            k = 6 if self.kind == "c5" else args.order
            if self.kind == "c5":
                c = synth.nedelec_order6_case(args.size or 12, mesh=mesh)
            else:
                c = synth.nedelec_slab_case(k, args.size or 24, mesh=mesh)
            self.family, self.degree = FFG_TETRA_NEDELEC, k
            self.v, self.t, self.cell_a = c.vertices, c.cells, c.cell_curl
            self.coef_a, self.coef_b = 1.0, c.mass
            self._src = c.source
            n = c.meta["n"]
            self.name = (f"nedelec_order{k}_{'slabs' if self.kind == 'c3' else 'stress'}_"
                         f"{n}cube_x6")
            self.desc = dict(order=k, mass=c.mass, quadrature="exact reference tensors")

    def source(self, points):
        return np.ascontiguousarray(self._src(points))

    # -- the oracle's FP64 pipeline (assemble, load, constraints, reduction)
    def oracle_system(self, samples, cells=None):
        oracle = _oracle()
        v, t = self.v, (self.t if cells is None else cells)
        if self.kind == "c2":
            ca = self.cell_a if cells is None else self.cell_a[: len(t)]
            n, cp, ri, val = oracle.lagrange_csc(v, t, 2, 1, 0, 1.0, 0.0, ca)
            b = oracle.lagrange_load_samples(v, t, 2, samples, 1, 0)
            con, _ = oracle.lagrange_dirichlet(2, v, t)
        elif self.kind == "c1":
            n, cp, ri, val = oracle.p1_csc(v, t, 0.0, 1.0)
            b = oracle.p1_load(v, t, 1.0)
            con = oracle.square_boundary(len(v), t)
        else:
            ca = self.cell_a if cells is None else self.cell_a[: len(t)]
            n, cp, ri, val = oracle.nedelec_csc(v, t, self.degree, 1.0, self.coef_b, ca, None)
            b = oracle.nedelec_load_samples(v, t, self.degree, samples)
            con = oracle.pec_mask(self.degree, t)
        return n, oracle.reduce_constrained(n, cp, ri, val, b, con)


# ---------------------------------------------------------------- CPU legs

def cpu_full(work, samples, max_iterations=400000):
    """The oracle's full FP64 pipeline on this host (1 core, the reference is
    serial): assembly, load, constraints, reduction and Jacobi-PCG to the
    reference's stopping rule, each phase timed."""
    oracle = _oracle()
    t0 = time.perf_counter()
    n, (nf, rcp, rri, rv, rr, free) = work.oracle_system(samples)
    t_asm = time.perf_counter() - t0
    t0 = time.perf_counter()
    x, s = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=TOL, max_iterations=max_iterations, guard=1)
    t_pcg = time.perf_counter() - t0
    r = rr - oracle.csc_matvec(nf, rcp, rri, rv, x)
    true = float(np.linalg.norm(r) / np.linalg.norm(rr))
    return dict(seconds=t_asm + t_pcg, assembly_s=t_asm, pcg_s=t_pcg, n_dofs=n, x=x, free=free,
                iterations=s["iterations"], converged=s["converged"], true_relative_residual=true)


def cpu_sampled(work, samples, reduced, n_iter, cell_fraction, pcg_iters=5):
    """A bounded sample of the oracle's FP64 pipeline, for systems whose full
    CPU solve takes hours: the assembly + load + constraints + reduction of
    the first `cell_fraction` of the cells scaled to all cells, plus
    `pcg_iters` oracle Jacobi-PCG iterations on the full reduced system
    (values from the GPU's FP64 assembly) scaled to `n_iter` iterations."""
    oracle = _oracle()
    m = max(1, int(len(work.t) * cell_fraction))
    sub = np.ascontiguousarray(work.t[:m])
    t0 = time.perf_counter()
    work.oracle_system(np.ascontiguousarray(samples[:m]), cells=sub)
    t_asm = (time.perf_counter() - t0) * len(work.t) / m
    R, rhs = reduced
    t0 = time.perf_counter()
    oracle.pcg_sparse(R.nrow, R.col_ptr, R.row_idx, R.val, rhs, tol=1e-300,
                      max_iterations=pcg_iters, guard=1)
    t_it = (time.perf_counter() - t0) / pcg_iters
    return dict(seconds=t_asm + n_iter * t_it, assembly_s=t_asm, iter_s=t_it, cells=m,
                n_iter=n_iter, pcg_iters=pcg_iters)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    oracle = _oracle()
    work = Workload(args, mesh=lambda n: (oracle.box_mesh([n, n, n]) if args.workload != "c1"
                                          else oracle.unit_square_mesh(n)))
    if work.kind == "c2":
        pts = oracle.lagrange_quadrature_points(work.v, work.t, 1, 0)
    elif work.kind == "c1":
        pts = work.v[work.t].mean(axis=1)[:, None, :]
        pts = np.concatenate([pts, np.zeros(pts.shape[:-1] + (1,))], -1)
    else:
        pts = oracle.nedelec_load_points(work.v, work.t, work.degree)
    samples = work.source(pts)
    if work.kind == "c1":
        samples = samples.reshape(-1)
    # setup: the reduced system and the reference PCG's iteration count
    n, (nf, rcp, rri, rv, rr, free) = work.oracle_system(samples)
    small = work.kind in ("c1",) or (work.kind == "c3" and work.degree == 1)
    if work.kind == "c2" or small:
        _, s = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=TOL, max_iterations=400000, guard=1)
        n_iter = s["iterations"]
    elif args.ref_iterations > 0:
        n_iter = args.ref_iterations
    else:
        print(json.dumps({"impl": "reference", "unavailable":
                          "the CPU FP64 Jacobi-PCG of this system runs for hours; pass "
                          "--ref-iterations (the GPU FP64 path's count) to time a bounded "
                          "sample"}), flush=True)
        return 0
    frac = 1.0 if (small or work.kind == "c2") else 0.02
    steps = []
    for i in range(args.warmup + args.steps):
        m = max(1, int(len(work.t) * (0.125 if work.kind == "c2" else frac)))
        sub = np.ascontiguousarray(work.t[:m])
        t0 = time.perf_counter()
        work.oracle_system(np.ascontiguousarray(samples[:m]), cells=sub)
        t_asm = (time.perf_counter() - t0) * len(work.t) / m
        t0 = time.perf_counter()
        oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=1e-300, max_iterations=10, guard=1)
        t_it = (time.perf_counter() - t0) / 10
        if i >= args.warmup:
            steps.append(t_asm + (n_iter or 0) * t_it)
    sec = float(np.mean(steps))
    value = n / sec
    sample = (f"per step: oracle assembly + load + constraints + reduction of "
              f"{'1/8 of the cells' if work.kind == 'c2' else 'all cells'} scaled to the mesh, "
              f"10 FP64 Jacobi-PCG iterations on the full reduced system scaled to {n_iter} "
              f"iterations (counted by one full CPU solve to 1e-10 in setup); mesh from the "
              f"oracle's Kuhn generator")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "DoF/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": work.name, "n_dofs": n, "solver": "fp64 jacobi-pcg"},
            "cpu_baseline": {"value": value, "unit": "DoF/s", "cores": 1, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "DoF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU leg

class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region; the raw
    samples go to clocks_<gpu>.csv in $FFG_CLOCKS_DIR (default: the temp dir)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        out = os.environ.get("FFG_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"clocks_{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def pcg_bytes(stats, nnz, nf, fp64_continuation, half=False):
    """Algorithmic bytes of one pcg_kernel launch: per FP32 inner iteration the
    FP32 SpMV with a 4-byte index plus eight FP32 vector streams (8 nnz + 44 n
    + 4; with the FP16 operator 6 nnz + 48 n + 4, the row scales included),
    per FP64 iteration or residual replacement the FP64 SpMV plus FP64 vectors
    (12 nnz + 4 (n + 1) + 32 n).  A solve that continued in FP64 is counted at
    the FP64 rate for all its iterations (an upper bound)."""
    inner = (6 * nnz + 48 * nf + 4) if half else (8 * nnz + 44 * nf + 4)
    outer = 12 * nnz + 4 * (nf + 1) + 32 * nf
    it = float(np.mean([s.iterations for s in stats]))
    ref = float(np.mean([s.refinements for s in stats]))
    if fp64_continuation:
        return (it + ref + 1) * outer
    return it * inner + (ref + 1) * outer


def run_ours(args):
    import torch
    import fortfem_b200 as ff

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)

    work = Workload(args)
    t0 = time.perf_counter()
    prob = ff.Problem(work.family, work.degree, work.t, len(work.v), rule=work.rule,
                      quadrature_degree=work.qdeg, boundary="all")
    setup_s = time.perf_counter() - t0
    if args.assembly == "tf32x3":
        prob.set_assembly_precision("tf32x3")
    pts = prob.sample_points(work.v)
    src = work.source(pts)
    if work.kind == "c1":
        src = np.ascontiguousarray(src.reshape(-1))   # f = 1 at the centroid
    tuning = None
    if args.autotune:
        tuning = prob.autotune(work.v, work.coef_a, work.coef_b, work.cell_a, work.cell_b, src)

    # inputs resident in HBM
    v_d = torch.from_numpy(np.ascontiguousarray(work.v)).to(dev)
    k_d = None if work.cell_a is None else torch.from_numpy(np.ascontiguousarray(work.cell_a)).to(dev)
    s_d = torch.from_numpy(np.ascontiguousarray(src)).to(dev)
    out_d = torch.zeros(prob.n_dofs, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    mixed = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=TOL,
                             precision=args.precision, max_iterations=args.max_iterations,
                             timeout_seconds=args.timeout)

    def step(opts=mixed):
        return prob.solve_device(v_d, out_d, work.coef_a, work.coef_b, k_d, None, s_d, None, opts,
                                 stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    per_step = []
    stats = []
    e0.record(stream)
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats.append(step())
        b.record(stream)
        per_step.append((a, b))
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    lat = [a.elapsed_time(b) for a, b in per_step]
    if dist:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    reached = max(s.true_relative_residual for s in stats)
    converged = all(s.converged and s.true_relative_residual <= TOL for s in stats)
    phases = prob.phase_times()
    value = world * prob.n_dofs * args.steps / (ms * 1e-3)
    sol = out_d.cpu().numpy()

    # roofline of the persistent PCG kernel (algorithmic bytes / kernel time)
    nnz, nf = prob.nnz, prob.n_free
    alg = pcg_bytes(stats, nnz, nf, phases["fp64_continuation"], args.precision == "mixed16")
    kt = float(np.mean([s.solve_time for s in stats]))
    peak, peak_kind = measured_peaks()
    achieved = alg / kt / 1e9
    traffic = None
    if work.kind == "c2" and (args.size or 48) == 48 and args.precision == "mixed":
        traffic = PCG_TRAFFIC_BYTES * alg / PCG_TRAFFIC_ALG_BYTES
    roofline = {"kernel": "pcg_kernel (persistent mixed Jacobi-PCG)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "traffic": traffic,
                "frac_dram": (traffic / kt / 1e9 / peak) if traffic else None,
                "algorithmic_bytes_per_launch": alg, "kernel_ms": kt * 1e3}

    # Nedelec: roofline of the assembly kernels (element matrices, loads and
    # the SELL gather) by their algorithmic bytes per assembly
    asm_roof = None
    if work.family == ff.FFG_TETRA_NEDELEC:
        gd = prob.topology()["global_dofs"]
        free = ~prob.constrained()
        inc = int(free[gd].sum())                    # (cell, local DoF) pairs on free DoFs
        T, nb = gd.shape
        nq = pts.shape[1]
        per_cell = (-(-nb * nb // 32) * 32) * 4 if args.assembly == "tf32x3" else nb * nb * 8
        alg_a = (2 * T * per_cell                    # element matrices written and gathered
                 + inc * nb * 2                      # slot rows
                 + nnz * 12                          # FP64 + FP32 operator values
                 + T * nq * 24 + T * nb * 8 + inc * 8)   # samples, element loads written / read
        at = float(np.mean([s.assembly_time for s in stats]))
        asm_roof = {"kernels": ("ort_matrix_kernel or nedelec_tc_kernel, ort_load_kernel, "
                                "sell_slice_kernel / column_kernel"),
                    "bound": "hbm", "achieved": alg_a / at / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": alg_a / at / 1e9 / peak, "peak_source": peak_kind,
                    "algorithmic_bytes": alg_a, "assembly_ms": at * 1e3}

    line = {"metric": METRIC, "value": value, "unit": "DoF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f32 SpMV/PCG + f64 geometry, assembly, residual, refinement" +
                      ("; 3xTF32 element contraction" if args.assembly == "tf32x3" else "")),
            "data": "synthetic",
            "config": {"workload": work.name, "cells": prob.n_cells, "n_dofs": prob.n_dofs,
                       "n_free": nf, "nnz_constrained": nnz, **work.desc,
                       "assembly": args.assembly,
                       "solver": ("mixed: FP32 Jacobi-PCG inner" +
                                  (" on a row-scaled FP16 operator" if args.precision == "mixed16"
                                   else "") + ", FP64 iterative refinement"),
                       "tolerance": TOL, "parallelism": f"replicas x{world}",
                       "l2": ("inputs larger than L2" if nnz * 12 > 126e6 else
                              "operator smaller than L2 (resident between steps)")},
            "converged": converged, "true_relative_residual": reached,
            "iterations": float(np.mean([s.iterations for s in stats])),
            "refinements": float(np.mean([s.refinements for s in stats])),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "assembly_ms": float(np.mean([s.assembly_time for s in stats])) * 1e3,
            "setup_seconds": setup_s, "roofline": roofline, "assembly_roofline": asm_roof,
            "clocks": clk,
            "pcg_phase_ms": {k: (v * 1e3 if not isinstance(v, bool) else v) for k, v in phases.items()},
            # per step: geometry + column gather + pcg + solution scatter; Nedelec:
            # matrix (or tensor-core) + load + gather + pcg + scatter
            "gpu_launches": (5 if work.family == ff.FFG_TETRA_NEDELEC else 4) * args.steps}
    if tuning:
        line["tuning"] = tuning
    if not converged:
        # where the solve stopped short of 1e-10: the FP64 rounding floor of b - A x
        R, rhs, free = prob.reduced_system(work.v, work.coef_a, work.coef_b, work.cell_a, None,
                                           src)
        import scipy.sparse as sp
        A = sp.csc_matrix((R.val, R.row_idx, R.col_ptr), shape=(R.nrow, R.nrow))
        xf = sol[free]
        line["fp64_floor"] = float(EPS * np.linalg.norm(abs(A) @ abs(xf)) / np.linalg.norm(rhs))
        line["stopped"] = ("true residual stopped falling above 1e-10; fp64_floor is "
                           "eps || |A| |x| || / ||b|| of the returned x")
        reduced = (R, rhs)
    else:
        reduced = None

    # plain FP64 GPU path (same kernels, FP64 values and vectors, no refinement)
    if not args.no_fp64:
        fp64 = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=TOL,
                                precision="fp64", breakdown_guard="spd",
                                max_iterations=args.max_iterations, timeout_seconds=args.timeout)
        step(fp64)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        n64 = max(1, min(args.steps, 3))
        a.record(stream)
        s64 = [step(fp64) for _ in range(n64)]
        b.record(stream)
        torch.cuda.synchronize()
        ms64 = a.elapsed_time(b) / n64
        line["fp64_gpu"] = {"value": prob.n_dofs / (ms64 * 1e-3), "unit": "DoF/s",
                            "ms_per_step": ms64, "iterations": s64[-1].iterations,
                            "converged": bool(s64[-1].converged),
                            "true_relative_residual": s64[-1].true_relative_residual}
        line["mixed_over_fp64"] = value / world / line["fp64_gpu"]["value"]

    # end to end through the host-array API with pinned host buffers
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        vh, sh = pin(work.v), pin(src)
        kh = None if work.cell_a is None else pin(work.cell_a)
        h2d = vh.nbytes + sh.nbytes + (0 if kh is None else kh.nbytes)
        d2h = prob.n_dofs * 8
        out_h = torch.zeros(prob.n_dofs, dtype=torch.float64).pin_memory().numpy()
        prob.solve(vh, work.coef_a, work.coef_b, kh, None, sh, None, mixed, out=out_h)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            prob.solve(vh, work.coef_a, work.coef_b, kh, None, sh, None, mixed, out=out_h)
        b.record()
        torch.cuda.synchronize()
        ems = a.elapsed_time(b)
        if dist:
            tt = torch.tensor([ems], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        line["e2e"] = {"value": world * prob.n_dofs * args.steps / (ems * 1e-3), "unit": "DoF/s",
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "ms_per_step": ems / args.steps}

    # serving: a Poisson stream of P1/P2 requests through the continuous-batching
    # server; with N GPUs the stream is N times longer and faster and each rank
    # serves its share (no exchange on the data path); latency from arrival to
    # solution on the host
    if args.serving_requests > 0:
        from fortfem_b200 import replicas, serving
        reqs = serving.poisson_stream(args.serving_requests * world, args.serving_rate * world,
                                      seed=4)
        share = replicas.partition_requests(reqs, world)[rank]
        res, wall, setup = serving.run_requests(share, device=local)
        rows = replicas.gather_lists([(r.rid, r.latency, r.converged, r.iterations,
                                       r.true_relative_residual, r.mode, r.batch_size,
                                       r.device_seconds) for r in res])
        res_all = [serving.Result(i, lt, cv, it, tr, mode, bs, None, dv)
                   for i, lt, cv, it, tr, mode, bs, dv in rows]
        res_all.sort(key=lambda r: r.rid)
        sv = serving.summarize(reqs, res_all, replicas.max_over_ranks(wall),
                               replicas.max_over_ranks(setup), args.serving_rate * world)
        sv.pop("results")
        line["serving"] = {k: sv[k] for k in (
            "requests", "rate_per_s", "wall_s", "setup_s", "latency_ms", "latency_ms_by_mode",
            "converged", "not_converged", "max_true_relative_residual", "free_dofs_per_s",
            "whole_device", "cta_groups", "mean_batch")}
        line["serving"]["workload"] = ("70% P1 unit square n ~ logU[32,1024] squares/side, "
                                       "30% P2 Kuhn box n ~ logU[8,40]; lognormal cell "
                                       "coefficient, GRF source (RFF, corr. length 0.1), "
                                       "Poisson arrivals; tolerance 1e-10 true residual; "
                                       "stream split over ranks by estimated work")

    if rank == 0 and world == 1 and not args.no_cpu:
        full_cpu = work.kind in ("c1", "c2") or (work.kind == "c3" and work.degree == 1)
        if full_cpu:
            cpu = cpu_full(work, src)
            xo = cpu["x"]
            line["cpu_baseline"] = {
                "value": cpu["n_dofs"] / cpu["seconds"], "unit": "DoF/s", "cores": 1,
                "kind": "port",
                "sample": (f"the whole step on one core, measured, no extrapolation: oracle "
                           f"assembly + load + constraints + reduction ({cpu['assembly_s']:.1f} "
                           f"s) and FP64 Jacobi-PCG to the reference's stopping rule "
                           f"({cpu['iterations']} iterations, {cpu['pcg_s']:.1f} s, true "
                           f"residual {cpu['true_relative_residual']:.2e})")}
            xg = sol[cpu["free"]]
            line["solution_rel_err_vs_oracle"] = float(np.linalg.norm(xg - xo) /
                                                       np.linalg.norm(xo))
            line["oracle_true_relative_residual"] = cpu["true_relative_residual"]
        else:
            if reduced is None:
                R, rhs, _ = prob.reduced_system(work.v, work.coef_a, work.coef_b, work.cell_a,
                                                None, src)
                reduced = (R, rhs)
            n_iter = line.get("fp64_gpu", {}).get("iterations") or int(line["iterations"])
            frac = 0.02 if work.kind == "c3" else 0.005
            cpu = cpu_sampled(work, src, reduced, n_iter, frac)
            line["cpu_baseline"] = {
                "value": prob.n_dofs / cpu["seconds"], "unit": "DoF/s", "cores": 1,
                "kind": "port",
                "sample": (f"oracle assembly + load + constraints + reduction of the first "
                           f"{cpu['cells']} cells scaled to {prob.n_cells} "
                           f"({cpu['assembly_s']:.1f} s), {cpu['pcg_iters']} oracle FP64 "
                           f"Jacobi-PCG iterations on the full reduced system "
                           f"({cpu['iter_s'] * 1e3:.1f} ms each) scaled to {n_iter} iterations "
                           f"(the GPU FP64 path's count); the full CPU solve takes hours")}
            line["solution_rel_err_vs_oracle"] = None
            line["solution_error_note"] = ("the oracle's full FP64 solve of this system takes "
                                           "hours on one core; see the size-reduced parity "
                                           "tests")
    prob.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
