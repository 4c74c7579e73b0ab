"""Benchmark: assembled+solved DoF/s at relative residual 1e-10 on the P2
tetrahedral Poisson workload (48^3 x 6 jittered Kuhn box, 663,552 cells,
912,673 DoFs, lognormal cell coefficient, sin*sin*sin source at the 4-point
rule, homogeneous Dirichlet).

One step = assemble (geometry + contraction + scatter + load + Dirichlet
reduction) + mixed-precision Jacobi-PCG until the true FP64 residual
||b - A x|| / ||b|| <= 1e-10, from inputs resident in HBM.  The topology
(DoF numbering, CSC pattern, slot maps) is built once per mesh and reported as
setup.  `e2e` repeats the step through the public host-array API with the
host<->device copies inside the timed region.  With --gpus N > 1 every rank
solves its own replica (the path has no exchange step for independent
systems); value = total DoFs solved / max over ranks of the time.

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
WORKLOAD = "p2_tetra_poisson_48cube_x6_jittered_lognormal"
TOL = 1e-10
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one pcg_kernel
# launch on the 48^3 workload, from an ncu capture of
# `bench.py --steps 1 --warmup 3 --no-cpu --no-e2e --no-fp64 --serving-requests 0`, and the
# algorithmic bytes of that launch; the live launch's traffic is scaled by
# its own algorithmic bytes.
PCG_TRAFFIC_BYTES = 101.803065e9 + 3.318534e9
PCG_TRAFFIC_ALG_BYTES = 159007138196.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=48)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=128,
                    help="requests of the serving leg (0 skips it)")
    ap.add_argument("--serving-rate", type=float, default=20.0)
    return ap.parse_args()


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


# ---------------------------------------------------------------- CPU legs

def cpu_reference_sample(case, n_iter=None, pcg_sample_iters=10):
    """Time the oracle's FP64 restatement of the reference path on this host (1 core):
    full-size assembly (DoF map, element loop, triplet->CSC), load, Dirichlet data
    and reduction, then `pcg_sample_iters` Jacobi-PCG iterations on the full
    reduced system, extrapolated to `n_iter` iterations.  When n_iter is None
    the CPU PCG is run to convergence once to count them."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    v, t, kappa = case.vertices, case.cells, case.cell_coefficient
    t0 = time.perf_counter()
    n, cp, ri, val = oracle.lagrange_csc(v, t, 2, 1, 0, 1.0, 0.0, kappa)
    t_asm = time.perf_counter() - t0
    pts = oracle.lagrange_quadrature_points(v, t, 1, 0)
    src = case.source(pts[..., 0], pts[..., 1], pts[..., 2])
    t0 = time.perf_counter()
    b = oracle.lagrange_load_samples(v, t, 2, src, 1, 0)
    con, _ = oracle.lagrange_dirichlet(2, v, t)
    nf, rcp, rri, rv, rr, free = oracle.reduce_constrained(n, cp, ri, val, b, con)
    t_bc = time.perf_counter() - t0
    counted = None
    if n_iter is None:
        t0 = time.perf_counter()
        _, s = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=TOL, max_iterations=200000, guard=1)
        t_full = time.perf_counter() - t0
        counted = s
        n_iter = s["iterations"]
        t_iter = t_full / max(n_iter, 1)
    else:
        t0 = time.perf_counter()
        oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=1e-300, max_iterations=pcg_sample_iters, guard=1)
        t_iter = (time.perf_counter() - t0) / pcg_sample_iters
    total = t_asm + t_bc + n_iter * t_iter
    return dict(seconds=total, n_dofs=n, assembly_s=t_asm, bc_s=t_bc, iter_s=t_iter, n_iter=n_iter,
                counted=counted, data=(nf, rcp, rri, rv, rr))


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from fortfem_b200 import synth
    case = synth.p2_poisson_case(args.size)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    # setup: one full CPU solve counts the FP64 Jacobi-PCG iterations to 1e-10
    full = cpu_reference_sample(case, None)
    nf, rcp, rri, rv, rr = full["data"]
    n_iter = full["n_iter"]
    steps = []
    v, t, kappa = case.vertices, case.cells, case.cell_coefficient
    sub = t[: max(len(t) // 8, 1)]
    pts = oracle.lagrange_quadrature_points(v, t, 1, 0)
    src = case.source(pts[..., 0], pts[..., 1], pts[..., 2])
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.lagrange_csc(v, sub, 2, 1, 0, 1.0, 0.0, kappa[: len(sub)])
        t_asm = (time.perf_counter() - t0) * (len(t) / len(sub))
        t0 = time.perf_counter()
        n, cp, ri, val = 0, None, None, None
        b = oracle.lagrange_load_samples(v, t, 2, src, 1, 0)
        con, _ = oracle.lagrange_dirichlet(2, v, t)
        t_bc = time.perf_counter() - t0
        t0 = time.perf_counter()
        oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=1e-300, max_iterations=10, guard=1)
        t_it = (time.perf_counter() - t0) / 10
        if i >= args.warmup:
            steps.append(t_asm + t_bc + full["bc_s"] * 0 + n_iter * t_it)
    sec = float(np.mean(steps))
    value = full["n_dofs"] / sec
    sample = (f"per step: oracle assembly of 1/8 of the cells scaled x8, full-size load + "
              f"Dirichlet data, 10 FP64 Jacobi-PCG iterations on the full reduced system scaled to "
              f"{n_iter} iterations (counted by one full CPU solve to 1e-10 in setup)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "DoF/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_dofs": full["n_dofs"], "solver": "fp64 jacobi-pcg"},
            "cpu_baseline": {"value": value, "unit": "DoF/s", "cores": 1, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "DoF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "full_cpu_solve_seconds": full["seconds"]}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU leg

def run_ours(args):
    import torch
    import fortfem_b200 as ff
    from fortfem_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)

    case = synth.p2_poisson_case(args.size)
    t0 = time.perf_counter()
    prob = ff.Problem(case.family, case.degree, case.cells, len(case.vertices), rule=case.rule,
                      quadrature_degree=case.quadrature_degree)
    setup_s = time.perf_counter() - t0
    pts = prob.sample_points(case.vertices)
    src = case.source(pts[..., 0], pts[..., 1], pts[..., 2])

    # inputs resident in HBM
    v_d = torch.from_numpy(case.vertices).to(dev)
    k_d = torch.from_numpy(case.cell_coefficient).to(dev)
    s_d = torch.from_numpy(np.ascontiguousarray(src)).to(dev)
    out_d = torch.zeros(prob.n_dofs, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    mixed = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=TOL,
                             precision="mixed", max_iterations=1000000, timeout_seconds=60)

    def step(opts=mixed):
        return prob.solve_device(v_d, out_d, 1.0, 0.0, k_d, None, s_d, None, opts, stream)

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
    converged = all(s.converged and s.true_relative_residual <= TOL for s in stats)
    phases = prob.phase_times()
    value = world * prob.n_dofs * args.steps / (ms * 1e-3)

    # roofline of the persistent PCG kernel (algorithmic bytes / kernel time)
    nnz, nf = prob.nnz, prob.n_free
    it = float(np.mean([s.iterations for s in stats]))
    ref = float(np.mean([s.refinements for s in stats]))
    bytes_inner = 8 * nnz + 44 * nf + 4          # FP32 SpMV + 8 FP32 vector streams
    bytes_outer = 12 * nnz + 4 * (nf + 1) + 32 * nf  # FP64 residual SpMV + FP64 vectors
    alg = it * bytes_inner + (ref + 1) * bytes_outer
    kt = float(np.mean([s.solve_time for s in stats]))
    peak, peak_kind = measured_peaks()
    achieved = alg / kt / 1e9
    roofline = {"kernel": "pcg_kernel (persistent mixed Jacobi-PCG)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind,
                "traffic": (PCG_TRAFFIC_BYTES * alg / PCG_TRAFFIC_ALG_BYTES
                            if args.size == 48 else None),
                "algorithmic_bytes_per_launch": alg, "kernel_ms": kt * 1e3}

    line = {"metric": METRIC, "value": value, "unit": "DoF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 SpMV/PCG + f64 geometry, assembly, residual, refinement",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": prob.n_cells, "n_dofs": prob.n_dofs,
                       "n_free": nf, "nnz_constrained": nnz, "degree": 2,
                       "quadrature": "4-point degree-two rule",
                       "solver": "mixed: FP32 Jacobi-PCG inner, FP64 iterative refinement",
                       "tolerance": TOL, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (FP64+FP32 CSC values and indices ~ 384 MB)"},
            "converged": converged,
            "iterations": it, "refinements": ref,
            "true_relative_residual": max(s.true_relative_residual for s in stats),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "assembly_ms": float(np.mean([s.assembly_time for s in stats])) * 1e3,
            "setup_seconds": setup_s, "roofline": roofline, "clocks": clk,
            "pcg_phase_ms": {k: (v * 1e3 if not isinstance(v, bool) else v) for k, v in phases.items()},
            "gpu_launches": 4 * args.steps}

    # plain FP64 GPU path (same kernels, FP64 values and vectors, no refinement)
    if not args.no_fp64:
        fp64 = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=TOL,
                                precision="fp64", breakdown_guard="spd", max_iterations=1000000,
                                timeout_seconds=60)
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
                            "true_relative_residual": s64[-1].true_relative_residual}
        line["mixed_over_fp64"] = value / world / line["fp64_gpu"]["value"]

    # end to end through the host-array API with pinned host buffers
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        vh, kh, sh = pin(case.vertices), pin(case.cell_coefficient), pin(src)
        h2d = vh.nbytes + kh.nbytes + sh.nbytes
        d2h = prob.n_dofs * 8
        out_h = torch.zeros(prob.n_dofs, dtype=torch.float64).pin_memory().numpy()
        prob.solve(vh, 1.0, 0.0, kh, None, sh, None, mixed, out=out_h)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            sol, _ = prob.solve(vh, 1.0, 0.0, kh, None, sh, None, mixed, out=out_h)
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
        res_all = [serving.Result(i, lat, cv, it, tr, mode, bs, None, dev)
                   for i, lat, cv, it, tr, mode, bs, dev in rows]
        res_all.sort(key=lambda r: r.rid)
        sv = serving.summarize(reqs, res_all, replicas.max_over_ranks(wall),
                               replicas.max_over_ranks(setup), args.serving_rate * world)
        sv.pop("results")
        line["serving"] = {k: sv[k] for k in (
            "requests", "rate_per_s", "wall_s", "setup_s", "latency_ms", "latency_ms_by_mode",
            "converged", "not_converged", "max_true_relative_residual", "free_dofs_per_s",
            "whole_device", "mean_batch")}
        line["serving"]["workload"] = ("70% P1 unit square n ~ logU[32,1024] squares/side, "
                                       "30% P2 Kuhn box n ~ logU[8,40]; lognormal cell "
                                       "coefficient, GRF source (RFF, corr. length 0.1), "
                                       "Poisson arrivals; tolerance 1e-10 true residual; "
                                       "stream split over ranks by estimated work")

    if rank == 0 and world == 1 and not args.no_cpu:
        n_iter = line.get("fp64_gpu", {}).get("iterations")
        cpu = cpu_reference_sample(case, n_iter)
        line["cpu_baseline"] = {
            "value": cpu["n_dofs"] / cpu["seconds"], "unit": "DoF/s", "cores": 1, "kind": "port",
            "sample": (f"full-size oracle assembly ({cpu['assembly_s']:.1f} s), load + Dirichlet "
                       f"+ reduction ({cpu['bc_s']:.1f} s), 10 FP64 Jacobi-PCG iterations "
                       f"({cpu['iter_s'] * 1e3:.1f} ms each) extrapolated to {cpu['n_iter']} "
                       f"iterations (the FP64 path's count on this system)")}
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
