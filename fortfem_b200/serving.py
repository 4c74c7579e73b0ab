"""Continuous-batching solve server for streams of independent Poisson requests.

fortfem solves one problem per call on the CPU; a GPU serving many requests
needs a loop around the same assemble + solve path.  Requests (P1 triangles or
P2 tetrahedra of different sizes) arrive over time.  The server keeps one
device-resident problem (topology, slot maps, solver workspace; one
``ffg_problem_create``) per mesh size, created while device memory allows and
released least-recently-used when it does not, and keeps launching work while
earlier work is still on the GPU:

* small systems (at most ``small_rows`` free DoFs) are packed into batches that
  are assembled together (one launch per phase) and solved one system per
  thread block in a single launch (``ffg_problem_solve_batch`` with
  ``FFG_BATCH_CTA_PER_SYSTEM``); up to ``streams`` such batches are in flight
  at once and overlap on the device;
* a large system runs on the whole GPU (``FFG_BATCH_WHOLE_DEVICE``), alone:
  its cooperative launch needs every SM, so it waits until the small batches
  in flight have drained, and no new batch starts until it is done.

Requests of one mesh size can share a batch and run in overlapping batches:
the engine keeps a pool of problems per size (each with its own workspace)
and grows it while memory allows.  Requests are served first come, first
served, except that small requests may run ahead of a waiting large one for
at most ``bypass_window`` seconds after the large one arrived; after that the
large request stops admission until the device has drained and it has run.

Each request carries only its seeds; its inputs (jittered vertices, lognormal
cell coefficients, a Gaussian-random-field source) are synthesized on the
device on the stream of its batch, so the host never holds per-request
arrays.  The solution is copied to pinned host memory before the request
counts as finished; latency runs from arrival to that point.

The scheduling logic (``Scheduler``) is separate from the device work
(``DeviceEngine``) so that it can be exercised without a GPU.
"""
from __future__ import annotations

import math
import time
from collections import Counter, deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from ._capi import FFG_RULE_DEGREE_TWO, FFG_TETRA_LAGRANGE, FFG_TRIANGLE_P1

# 4-point degree-two rule (reference coordinates, the order of the library's rule)
_A2 = (5.0 + 3.0 * math.sqrt(5.0)) / 20.0
_B2 = (5.0 - math.sqrt(5.0)) / 20.0
DEGREE_TWO_POINTS = ((_B2, _B2, _B2), (_A2, _B2, _B2), (_B2, _A2, _B2), (_B2, _B2, _A2))


@dataclass
class Request:
    """One Poisson solve: family "p1" (n x n squares, 2 triangles each) or
    "p2" (n^3 hexes, 6 tetrahedra each), with its seed and arrival time (s)."""
    rid: int
    family: str
    n: int
    seed: int
    arrival: float = 0.0

    @property
    def key(self) -> Tuple[str, int]:
        return (self.family, self.n)


@dataclass
class Result:
    rid: int
    latency: float
    converged: bool
    iterations: int
    true_relative_residual: float
    mode: str
    batch_size: int
    solution: Optional[np.ndarray] = None
    device_seconds: float = 0.0   # its assembly + the solve of its batch, on the device


def poisson_stream(count: int, rate: float, seed: int = 4, p1_fraction: float = 0.7,
                   p1_range=(32, 1024), p2_range=(8, 40)) -> List[Request]:
    """Poisson arrivals at `rate` per second; sizes log-uniform in the ranges."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
    is_p1 = rng.random(count) < p1_fraction
    u = rng.random(count)
    out = []
    for i in range(count):
        lo, hi = p1_range if is_p1[i] else p2_range
        n = int(round(math.exp(math.log(lo) + u[i] * (math.log(hi) - math.log(lo)))))
        out.append(Request(i, "p1" if is_p1[i] else "p2", n, int(rng.integers(1, 2**31 - 1)),
                           float(arrivals[i])))
    return out


def free_dofs(key: Tuple[str, int]) -> int:
    """Free DoFs of a request's system (homogeneous Dirichlet on the boundary)."""
    family, n = key
    return (n - 1) ** 2 if family == "p1" else (2 * n - 1) ** 3


# --------------------------------------------------------------- scheduling

@dataclass
class Batch:
    mode: str                    # "cta_per_system" or "whole_device"
    requests: List[Request]
    slot: int                    # stream slot (whole-device batches use slot 0)
    token: object = None         # engine handle of the launched work


@dataclass
class Scheduler:
    """Decides which queued requests form the next batch (no device work)."""
    small_rows: int = 32768
    max_batch: int = 48
    streams: int = 2
    bypass_window: float = 0.05
    # large requests side by side in one cooperative launch ("cta_groups"),
    # each on group_ctas(key) of `grid` thread blocks, instead of one after
    # another on the whole device
    groups: bool = False
    grid: int = 148
    group_rows: int = 16384
    max_groups: int = 16
    queue: deque = field(default_factory=deque)
    inflight: List[Batch] = field(default_factory=list)

    def is_small(self, r: Request) -> bool:
        return free_dofs(r.key) <= self.small_rows

    def group_ctas(self, key) -> int:
        """Thread blocks of a system in a group launch (ffg_problem_solve_batch's
        FFG_BATCH_CTA_GROUPS rule: group_rows rows per block, 2 to grid)."""
        return max(2, min(-(-free_dofs(key) // self.group_rows), self.grid))

    def _large_batch(self, head: Request, can_host) -> Batch:
        picked, counts = [head], Counter({head.key: 1})
        used = self.group_ctas(head.key)
        if self.groups:
            for r in list(self.queue)[1:]:
                if len(picked) == self.max_groups:
                    break
                if self.is_small(r):
                    continue
                g = self.group_ctas(r.key)
                if used + g > self.grid or not can_host(r.key, counts[r.key] + 1):
                    continue
                picked.append(r)
                counts[r.key] += 1
                used += g
        for r in picked:
            self.queue.remove(r)
        return Batch("cta_groups" if self.groups else "whole_device", picked, 0)

    def busy_counts(self) -> Counter:
        return Counter(r.key for b in self.inflight for r in b.requests)

    def _starved(self, r: Request, now) -> bool:
        return now is None or now - r.arrival >= self.bypass_window

    def next_batch(self, can_host, now: Optional[float] = None) -> Optional[Batch]:
        """The batch to launch now, or None.  `can_host(key, count)` says
        whether the engine can provide `count` problems of that mesh size at
        once; `now` (seconds, the arrivals' clock) lets small requests pass a
        large one that has waited less than bypass_window (without it the
        queue is strictly first come, first served)."""
        if not self.queue:
            return None
        if any(b.mode != "cta_per_system" for b in self.inflight):
            return None
        head = self.queue[0]
        if not self.is_small(head):
            if not self.inflight and can_host(head.key, 1):
                return self._large_batch(head, can_host)
            if self._starved(head, now):
                return None
        used = {b.slot for b in self.inflight}
        free_slots = [s for s in range(self.streams) if s not in used]
        if not free_slots:
            return None
        busy = self.busy_counts()
        picked, counts = [], Counter()
        for r in self.queue:
            if not self.is_small(r):
                if self._starved(r, now):
                    break
                continue
            if not can_host(r.key, busy[r.key] + counts[r.key] + 1):
                continue
            picked.append(r)
            counts[r.key] += 1
            if len(picked) == self.max_batch:
                break
        if not picked:
            return None
        for r in picked:
            self.queue.remove(r)
        return Batch("cta_per_system", picked, free_slots[0])


def percentiles(latencies: List[float]) -> Dict[str, float]:
    a = np.asarray(latencies) * 1e3
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
            "p99.9": float(np.percentile(a, 99.9)), "mean": float(a.mean()),
            "max": float(a.max())}


def serve(requests: List[Request], engine, scheduler: Optional[Scheduler] = None,
          clock=time.perf_counter, idle_sleep: float = 2e-5) -> List[Result]:
    """Replay `requests` (sorted by arrival) against `engine` in real time."""
    sch = scheduler or Scheduler()
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    results: List[Result] = []
    t0 = clock()
    while pending or sch.queue or sch.inflight:
        now = clock() - t0
        while pending and pending[0].arrival <= now:
            sch.queue.append(pending.popleft())
        for b in list(sch.inflight):
            if engine.done(b.token):
                t_done = clock() - t0
                for r, res in zip(b.requests, engine.collect(b.token)):
                    res.latency = t_done - r.arrival
                    res.mode, res.batch_size = b.mode, len(b.requests)
                    results.append(res)
                sch.inflight.remove(b)
        launched = False
        while True:
            b = sch.next_batch(engine.can_host, clock() - t0)
            if b is None:
                break
            b.token = engine.launch(b)
            sch.inflight.append(b)
            launched = True
        if not launched:
            if not sch.inflight and not sch.queue and pending:
                wait = pending[0].arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            else:
                time.sleep(idle_sleep)
    results.sort(key=lambda r: r.rid)
    return results


# ------------------------------------------------------------ device engine

class _Mesh:
    """Host topology and device-side templates of one mesh size."""

    def __init__(self, key, device):
        import torch
        from . import api, synth
        family, n = key
        self.key = key
        if family == "p1":
            v, t = api.unit_square_mesh(n + 1)
            self.problem = api.Problem(FFG_TRIANGLE_P1, 1, t, len(v), boundary="all")
            self.dim = 2
        else:
            v, t = synth.box_mesh(n)
            self.problem = api.Problem(FFG_TETRA_LAGRANGE, 2, t, len(v), rule=FFG_RULE_DEGREE_TWO,
                                       boundary="all")
            self.dim = 3
        self.h = 1.0 / n
        self.n_cells = len(t)
        self.base = torch.from_numpy(np.ascontiguousarray(v)).to(device)
        inner = np.all((v > 1e-12) & (v < 1 - 1e-12), axis=1)
        self.inner = torch.from_numpy(inner).to(device)
        self.cells = torch.from_numpy(np.ascontiguousarray(t, dtype=np.int64)).to(device)


class DeviceEngine:
    """Runs batches with the library on one GPU; inputs synthesized on the device.

    Per request: vertices jittered uniformly by +-0.1h off the boundary, cell
    coefficient exp(N(0,1)), source a Gaussian random field of correlation
    length 0.1 by `features` random Fourier features (sampled at the cell
    centroid for P1, at the 4 points of the degree-two rule for P2),
    homogeneous Dirichlet data.  Each solve has a 10 s device time limit so
    that one pathological request cannot hold the GPU."""

    def __init__(self, device: int = 0, memory_fraction: float = 0.8, options=None,
                 keep_solutions: bool = False, features: int = 64, corr_length: float = 0.1,
                 streams: int = 2, max_instances: int = 8):
        import torch
        from .api import SolverOptions
        self.torch = torch
        self.device = torch.device("cuda", device)
        free, _ = torch.cuda.mem_get_info(self.device)
        self.budget = int(free * memory_fraction)
        self.used = 0
        # a pool of problems per mesh size; `idle` holds the ones not in flight
        self.meshes: Dict[Tuple[str, int], List[_Mesh]] = {}
        self.idle: Dict[Tuple[str, int], List[_Mesh]] = {}
        self.bytes: Dict[Tuple[str, int], int] = {}
        self.last_use: Dict[Tuple[str, int], float] = {}
        self.max_instances = max_instances
        self.options = options or SolverOptions(method="pcg", preconditioner="jacobi",
                                                tolerance=1e-10, precision="mixed",
                                                max_iterations=1000000, timeout_seconds=10)
        self.keep = keep_solutions
        self.features = features
        self.corr = corr_length
        self.streams = [torch.cuda.Stream(self.device) for _ in range(streams)]
        self.setup_seconds = 0.0

    # -- problems per mesh size, admitted by device memory
    def _create(self, key):
        torch = self.torch
        t0 = time.perf_counter()
        torch.cuda.synchronize(self.device)
        before, _ = torch.cuda.mem_get_info(self.device)
        m = _Mesh(key, self.device)
        torch.cuda.synchronize(self.device)
        after, _ = torch.cuda.mem_get_info(self.device)
        self.meshes.setdefault(key, []).append(m)
        self.idle.setdefault(key, []).append(m)
        b = max(before - after, 0)
        self.bytes[key] = self.bytes.get(key, 0) + b
        self.used += b
        self.setup_seconds += time.perf_counter() - t0
        return m

    def _estimate(self, key) -> int:
        # bytes per free DoF seen so far for this family (P2 about 2.5 KB, P1 about 0.4 KB)
        same = [(k, b / len(self.meshes[k])) for k, b in self.bytes.items()
                if k[0] == key[0] and b > 0 and self.meshes.get(k)]
        per = (sum(b for _, b in same) / sum(free_dofs(k) for k, _ in same)) if same else \
            (2500.0 if key[0] == "p2" else 400.0)
        return int(per * free_dofs(key)) + (64 << 20)

    def _evict_for(self, need: int, keep=frozenset()) -> bool:
        # whole pools of sizes with nothing in flight, least recently used
        # first, sparing the sizes in `keep`
        idle = sorted((k for k, ms in self.meshes.items()
                       if k not in keep and len(self.idle.get(k, [])) == len(ms)),
                      key=lambda k: self.last_use.get(k, 0.0))
        for k in idle:
            if self.used + need <= self.budget:
                break
            for m in self.meshes.pop(k):
                m.problem.close()
            self.idle.pop(k, None)
            self.used -= self.bytes.pop(k)
        return self.used + need <= self.budget

    def can_host(self, key, count: int = 1, keep=frozenset()) -> bool:
        """Whether `count` problems of this mesh size can be in flight at
        once, creating pool members while memory allows (evicting idle pools
        of other sizes than `key` and those in `keep`)."""
        if count > self.max_instances:
            return False
        while len(self.meshes.get(key, [])) < count:
            need = self._estimate(key)
            if self.used + need > self.budget and not self._evict_for(need, keep | {key}):
                return False
            self._create(key)
        return True

    def prepare(self, requests: List[Request]) -> float:
        """Create the problems of every mesh size in `requests` ahead of time
        (as memory allows); returns the seconds spent (setup, not latency)."""
        t0 = self.setup_seconds
        for key in sorted({r.key for r in requests}, key=free_dofs):
            self.can_host(key)
        return self.setup_seconds - t0

    # -- device-side synthesis of a request's inputs
    def _inputs(self, m: _Mesh, r: Request):
        torch = self.torch
        g = torch.Generator(device=self.device)
        g.manual_seed(r.seed)
        d = m.dim
        jit = (torch.rand(m.base.shape, generator=g, device=self.device, dtype=torch.float64)
               * 2.0 - 1.0) * (0.1 * m.h)
        v = m.base + jit * m.inner[:, None].to(torch.float64)
        kappa = torch.exp(torch.randn(m.n_cells, generator=g, device=self.device,
                                      dtype=torch.float64))
        cv = v[m.cells]                                   # (T, d+1, d)
        if r.family == "p1":
            pts = cv.mean(dim=1)                          # (T, 2): one sample per cell
        else:
            xi = torch.tensor(DEGREE_TWO_POINTS, device=self.device, dtype=torch.float64)
            e = cv[:, 1:, :] - cv[:, :1, :]               # (T, 3, 3) edge vectors
            pts = cv[:, :1, :] + torch.einsum("qk,tkr->tqr", xi, e)   # (T, 4, 3)
            pts = pts.reshape(-1, 3)
        M = self.features
        omega = torch.randn((d, M), generator=g, device=self.device,
                            dtype=torch.float64) / self.corr
        phase = torch.rand(M, generator=g, device=self.device, dtype=torch.float64) * (2 * math.pi)
        amp = torch.randn(M, generator=g, device=self.device, dtype=torch.float64)
        src = torch.cos(pts @ omega + phase) @ amp * math.sqrt(2.0 / M)
        return v.contiguous(), kappa.contiguous(), src.contiguous()

    def launch(self, b: Batch):
        torch = self.torch
        from .api import solve_batch
        s = self.streams[b.slot]
        # a size admitted while the batch was formed may have been evicted
        # for a later one: host every size of the batch, sparing the others
        keep = frozenset(r.key for r in b.requests)
        for k, c in Counter(r.key for r in b.requests).items():
            busy = len(self.meshes.get(k, [])) - len(self.idle.get(k, []))
            if not self.can_host(k, busy + c, keep):
                raise RuntimeError(f"no device memory for {c} problems of size {k}")
        meshes = [self.idle[r.key].pop() for r in b.requests]
        for r in b.requests:
            self.last_use[r.key] = time.perf_counter()
        with torch.cuda.stream(s):
            ins = [self._inputs(m, r) for m, r in zip(meshes, b.requests)]
            sols = [torch.empty(m.problem.n_dofs, dtype=torch.float64, device=self.device)
                    for m in meshes]
            solve_batch([m.problem for m in meshes], [x[0] for x in ins], sols,
                        [1.0] * len(meshes), [0.0] * len(meshes), cell_a=[x[1] for x in ins],
                        samples=[x[2] for x in ins], options=self.options, mode=b.mode, stream=s)
            host = [torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for x in sols]
            for h, x in zip(host, sols):
                h.copy_(x, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        return (ev, meshes, host, ins, sols, b.requests)

    def done(self, token) -> bool:
        return token[0].query()

    def collect(self, token) -> List[Result]:
        ev, meshes, host, ins, sols, reqs = token
        out = []
        for m, h, r in zip(meshes, host, reqs):
            st = m.problem.batch_stats()
            self.idle[r.key].append(m)
            out.append(Result(r.rid, 0.0, bool(st.converged), st.iterations,
                              st.true_relative_residual, "", 0, h.numpy() if self.keep else None,
                              st.assembly_time + st.solve_time))
        return out

    def close(self):
        for ms in self.meshes.values():
            for m in ms:
                m.problem.close()
        self.meshes.clear()
        self.idle.clear()


def run_requests(reqs: List[Request], small_rows: int = 32768, max_batch: int = 48,
                 streams: int = 2, keep_solutions: bool = False, device: int = 0,
                 groups: bool = True):
    """Serve `reqs` (arrival times relative to now) on one GPU; returns
    (results, wall seconds, setup seconds).  Large requests run side by side
    in CTA groups (`groups`) or one after another on the whole device."""
    import torch
    eng = DeviceEngine(device, keep_solutions=keep_solutions, streams=streams)
    setup = eng.prepare(reqs)
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    sch = Scheduler(small_rows=small_rows, max_batch=max_batch, streams=streams, groups=groups,
                    grid=sms)
    t0 = time.perf_counter()
    res = serve(reqs, eng, sch) if reqs else []
    wall = time.perf_counter() - t0
    eng.close()
    return res, wall, setup


def summarize(reqs: List[Request], res: List[Result], wall: float, setup: float,
              rate: float) -> dict:
    """Latency percentiles (overall and per mode), convergence and throughput."""
    dofs = sum(free_dofs(r.key) for r in reqs)
    by_id = {r.rid: r for r in reqs}
    by_mode = {}
    for mode in ("cta_per_system", "whole_device", "cta_groups"):
        lat = [r.latency for r in res if r.mode == mode]
        if lat:
            by_mode[mode] = {"requests": len(lat), **percentiles(lat),
                             "device_s": float(sum(r.device_seconds for r in res
                                                   if r.mode == mode))}
    return {"requests": len(reqs), "rate_per_s": rate, "wall_s": wall, "setup_s": setup,
            "latency_ms": percentiles([r.latency for r in res]), "latency_ms_by_mode": by_mode,
            "converged": sum(r.converged for r in res),
            "max_true_relative_residual": max(r.true_relative_residual for r in res),
            "not_converged": [(by_id[r.rid].family, by_id[r.rid].n, r.true_relative_residual)
                              for r in res if not r.converged],
            "free_dofs_per_s": dofs / wall,
            "whole_device": sum(r.mode == "whole_device" for r in res),
            "cta_groups": sum(r.mode == "cta_groups" for r in res),
            "mean_batch": float(np.mean([r.batch_size for r in res])), "results": res}


def run_stream(count: int = 512, rate: float = 20.0, seed: int = 4, small_rows: int = 32768,
               max_batch: int = 48, streams: int = 2, keep_solutions: bool = False,
               device: int = 0, groups: bool = True) -> dict:
    """Serve a Poisson stream end to end on one GPU; returns latency statistics."""
    reqs = poisson_stream(count, rate, seed)
    res, wall, setup = run_requests(reqs, small_rows, max_batch, streams, keep_solutions, device,
                                    groups)
    return summarize(reqs, res, wall, setup, rate)


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="serve a stream of Poisson requests on one GPU")
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--small-rows", type=int, default=32768)
    ap.add_argument("--streams", type=int, default=2)
    ap.add_argument("--no-groups", action="store_true",
                    help="large requests one after another on the whole device")
    a = ap.parse_args()
    out = run_stream(a.requests, a.rate, a.seed, a.small_rows, streams=a.streams,
                     groups=not a.no_groups)
    out.pop("results")
    print(json.dumps(out))
