"""One system over several GPUs: owner-computes assembly and row-block
Jacobi-PCG with one halo exchange per iteration.

The reference solves a system on one CPU core; sharding is this library's
own extension.  The plan:

* cells are split into `world` parts by recursive coordinate bisection of
  their centroids; a free DoF belongs to the part of the first cell (in cell
  order) that contains it, so ownership is deterministic;
* rank r assembles, as an ordinary problem of its own, every cell that
  touches a DoF it owns (its owned cells plus one ghost layer).  The rows it
  owns are then complete - every element contribution to them is present -
  so assembly needs no reduction and each owned row equals the row of the
  single-GPU system, term for term;
* the iteration is the FP64 Jacobi-PCG of the single-GPU solver
  (advanced_solvers.f90:831-925 semantics: stop when ||r|| <= tol ||r_0||),
  with q = A p computed on every local row, dot products taken over owned
  rows only and all-reduced, and the new search direction of the ghost rows
  received from their owners before the next product (one exchange of the
  boundary entries of p per iteration).

Vectors of a rank live in device memory in the SELL row order of its
problem.  The exchange and the scalar all-reduces use torch.distributed:
NCCL on GPUs, gloo for CPU ranks; a CUDA rank under gloo stages the halo
through host memory.  The arithmetic runs in the library's kernels
(`DeviceOps`); no collective or kernel waits on another rank's kernel.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _capi as K
from .api import FortfemError, Problem, build_topology


def partition_cells(vertices, cells, parts: int) -> np.ndarray:
    """Owner part (0..parts-1) of every cell: recursive coordinate bisection of
    the cell centroids, splitting the longest extent at the weighted median
    (cell index breaks ties), so the result is deterministic."""
    v = np.asarray(vertices, float).reshape(-1, 3)
    t = np.asarray(cells).reshape(-1, 4)
    cen = v[t].mean(axis=1)
    owner = np.zeros(len(t), np.int32)

    def split(idx, lo, n):
        if n == 1 or len(idx) == 0:
            owner[idx] = lo
            return
        left = n // 2
        pts = cen[idx]
        ax = int(np.argmax(pts.max(axis=0) - pts.min(axis=0))) if len(idx) > 1 else 0
        order = idx[np.lexsort((idx, pts[:, ax]))]
        cut = (len(order) * left) // n
        split(order[:cut], lo, left)
        split(order[cut:], lo + left, n - left)

    split(np.arange(len(t)), 0, int(parts))
    return owner


@dataclass
class RankPlan:
    """What rank `rank` assembles and exchanges.  Row numbers below are the
    free-DoF indices of the rank's own problem (its submesh)."""
    rank: int
    world: int
    cells: np.ndarray          # global ids of the submesh cells, ascending
    vertex_ids: np.ndarray     # global ids of the submesh vertices, ascending
    sub_cells: np.ndarray      # submesh connectivity in local vertex ids
    constrained: np.ndarray    # uint8 mask over the submesh DoFs
    sub_to_global_free: np.ndarray  # submesh free index -> global free index
    sub_to_global_dof: np.ndarray   # submesh DoF -> global DoF
    owned: np.ndarray          # bool per submesh free index
    n_dofs: int = 0            # global DoF count
    free_dofs: np.ndarray = None    # global free index -> global DoF (shared by all plans)
    send: Dict[int, np.ndarray] = field(default_factory=dict)  # peer -> submesh free rows
    recv: Dict[int, np.ndarray] = field(default_factory=dict)  # peer -> submesh free rows


def build_plans(family: int, degree: int, vertices, cells, world: int, boundary="all",
                owner_of_cell: Optional[np.ndarray] = None) -> List[RankPlan]:
    """Plans of all `world` ranks (every rank computes the same list)."""
    vpc = 3 if family == K.FFG_TRIANGLE_P1 else 4
    cells = np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1, vpc))
    v = np.asarray(vertices, float)
    nv = len(v.reshape(-1, 3 if vpc == 4 else 2))
    if vpc != 4:
        raise FortfemError(K.FFG_INVALID_INPUT, "sharding covers the tetrahedral families")
    topo = build_topology(family, degree, cells, nv, boundary)
    gd = topo["global_dofs"]
    con = topo["constrained"]
    nd = topo["n_dofs"]
    free_index = np.full(nd, -1, np.int64)
    free = np.flatnonzero(~con)
    free_index[free] = np.arange(len(free))
    owner_cell = partition_cells(v, cells, world) if owner_of_cell is None else \
        np.asarray(owner_of_cell, np.int32)
    # a DoF belongs to the owner of the first cell that contains it
    first = np.full(nd, len(cells), np.int64)
    flat_c = np.repeat(np.arange(len(cells)), gd.shape[1])
    np.minimum.at(first, gd.ravel(), flat_c)
    dof_owner = owner_cell[first]
    plans = []
    for r in range(world):
        mine = (dof_owner == r) & ~con
        touch = np.flatnonzero(mine[gd].any(axis=1))
        vids = np.unique(cells[touch].ravel())
        local = np.full(nv, -1, np.int64)
        local[vids] = np.arange(len(vids))
        sub_cells = local[cells[touch]].astype(np.int32)
        # the submesh numbering, mapped DoF by DoF through the cells' local DoFs
        sub = build_topology(family, degree, sub_cells, len(vids), "none")
        sgd = sub["global_dofs"]
        s2g = np.full(sub["n_dofs"], -1, np.int64)
        s2g[sgd.ravel()] = gd[touch].ravel()
        scon = con[s2g].astype(np.uint8)
        sfree = np.flatnonzero(scon == 0)
        s2gf = free_index[s2g[sfree]]
        plans.append(RankPlan(rank=r, world=world, cells=touch, vertex_ids=vids,
                              sub_cells=sub_cells, constrained=scon, sub_to_global_free=s2gf,
                              sub_to_global_dof=s2g, owned=dof_owner[s2g[sfree]] == r,
                              n_dofs=nd, free_dofs=free))
    # ghost rows of r owned by s: r receives them from s, in global order
    owner_free = dof_owner[free]
    for p in plans:
        ghost = np.flatnonzero(~p.owned)
        g_glob = p.sub_to_global_free[ghost]
        for s in np.unique(owner_free[g_glob]):
            sel = owner_free[g_glob] == s
            order = np.argsort(g_glob[sel], kind="stable")
            p.recv[int(s)] = ghost[sel][order]
    for p in plans:
        pos = {int(g): i for i, g in enumerate(p.sub_to_global_free)}
        for q in plans:
            if p.rank in q.recv:
                need = q.sub_to_global_free[q.recv[p.rank]]
                p.send[q.rank] = np.array([pos[int(g)] for g in need], np.int64)
    return plans


# ------------------------------------------------------------------ device ops

def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class DeviceOps:
    """The rank's problem on its GPU: assembly, FP64 SpMV and the fused
    vector kernels of libfortfem_gpu (vectors are torch CUDA tensors in the
    problem's SELL row order)."""

    def __init__(self, plan: RankPlan, family: int, degree: int, rule: int, quadrature_degree: int,
                 device):
        import torch
        self.torch = torch
        self.device = device
        self.problem = Problem(family, degree, plan.sub_cells, len(plan.vertex_ids), rule=rule,
                               quadrature_degree=quadrature_degree, boundary=plan.constrained)
        n = self.problem.n_free
        perm = np.zeros(n, np.int32)
        st = C.c_int(0)
        K.load().ffg_problem_sell_permutation(self.problem.handle, perm.ctypes.data_as(C.c_void_p),
                                              C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_sell_permutation")
        self.row_of_free = np.empty(n, np.int64)
        self.row_of_free[perm] = np.arange(n)   # submesh free index -> SELL row
        self.n = n
        self.stream = None
        f64 = dict(dtype=torch.float64, device=device)
        self.work = torch.zeros(K.FFG_DIST_WORK_DOUBLES, **f64)
        self.dots = torch.zeros(4, **f64)

    def tensor(self, a, dtype=None):
        t = self.torch
        return t.as_tensor(np.ascontiguousarray(a), dtype=dtype or t.float64, device=self.device)

    def zeros(self, n):
        return self.torch.zeros(max(n, 1), dtype=self.torch.float64, device=self.device)

    def _check(self, st, where):
        if st.value:
            raise FortfemError(st.value, where)

    def assemble(self, vertices, coef_a, coef_b, cell_a, cell_b, samples, g):
        p = self.problem
        v, ca, cb, s, gg = p._inputs(vertices, cell_a, cell_b, samples, g)
        from .api import _ptr
        st = C.c_int(0)
        K.load().ffg_problem_assemble(p.handle, _ptr(v), float(coef_a), float(coef_b), _ptr(ca),
                                      _ptr(cb), _ptr(s), _ptr(gg), 0, None, C.byref(st))
        self._check(st, "ffg_problem_assemble")
        self.b = self.zeros(self.n)
        self.dinv = self.zeros(self.n)
        K.load().ffg_problem_system_arrays(p.handle, _p(self.b), _p(self.dinv), 1, None,
                                           C.byref(st))
        self._check(st, "ffg_problem_system_arrays")

    def spmv(self, x, y):
        st = C.c_int(0)
        K.load().ffg_problem_sell_spmv(self.problem.handle, _p(x), _p(y), None, C.byref(st))
        self._check(st, "ffg_problem_sell_spmv")

    def start(self, owned, ax, r, z, p):
        st = C.c_int(0)
        K.load().ffg_dist_start(self.n, _p(owned), _p(self.b), _p(ax), _p(self.dinv), _p(r),
                                _p(z), _p(p), _p(self.work), _p(self.dots), None, C.byref(st))
        self._check(st, "ffg_dist_start")
        return self.dots[:3].cpu().numpy().copy()

    def update(self, owned, alpha, p, q, x, r, z):
        st = C.c_int(0)
        K.load().ffg_dist_update(self.n, _p(owned), float(alpha), _p(p), _p(q), _p(self.dinv),
                                 _p(x), _p(r), _p(z), _p(self.work), _p(self.dots), None,
                                 C.byref(st))
        self._check(st, "ffg_dist_update")
        return self.dots[:2].cpu().numpy().copy()

    def dot(self, owned, a, b):
        st = C.c_int(0)
        K.load().ffg_dist_dot(self.n, _p(owned), _p(a), _p(b), _p(self.work), _p(self.dots),
                              None, C.byref(st))
        self._check(st, "ffg_dist_dot")
        return float(self.dots[0].item())

    def cgs_dots(self, owned, r, z, w):
        st = C.c_int(0)
        K.load().ffg_dist_cgs_dots(self.n, _p(owned), _p(r), _p(z), _p(w), _p(self.work),
                                   _p(self.dots), None, C.byref(st))
        self._check(st, "ffg_dist_cgs_dots")
        return self.dots[:3].cpu().numpy().copy()

    def cgs_update(self, owned, alpha, beta, w, p, s, x, r, z):
        st = C.c_int(0)
        K.load().ffg_dist_cgs_update(self.n, _p(owned), float(alpha), float(beta), _p(w),
                                     _p(self.dinv), _p(p), _p(s), _p(x), _p(r), _p(z), None,
                                     C.byref(st))
        self._check(st, "ffg_dist_cgs_update")

    def direction(self, owned, beta, z, p):
        st = C.c_int(0)
        K.load().ffg_dist_direction(self.n, _p(owned), float(beta), _p(z), _p(p), None,
                                    C.byref(st))
        self._check(st, "ffg_dist_direction")

    def gather(self, idx, src, dst):
        st = C.c_int(0)
        K.load().ffg_dist_gather(int(idx.numel()), _p(idx), _p(src), _p(dst), None, C.byref(st))
        self._check(st, "ffg_dist_gather")

    def scatter(self, idx, src, dst):
        st = C.c_int(0)
        K.load().ffg_dist_scatter(int(idx.numel()), _p(idx), _p(src), _p(dst), None, C.byref(st))
        self._check(st, "ffg_dist_scatter")

    def synchronize(self):
        self.torch.cuda.synchronize(self.device)

    def close(self):
        self.problem.close()


# --------------------------------------------------------------- the solver

@dataclass
class ShardStats:
    iterations: int = 0
    converged: bool = False
    final_residual: float = 0.0
    initial_residual: float = 0.0
    exchanged_values: int = 0
    allreduces: int = 0


class ShardedSolver:
    """Row-block Jacobi-PCG of one system on this rank.  `ops` computes on the
    rank's device (DeviceOps); every rank of the process group calls solve()
    with the same arguments."""

    def __init__(self, plan: RankPlan, ops, group=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.plan, self.ops, self.group = plan, ops, group
        rows = ops.row_of_free
        dev = ops.device
        owned_rows = np.zeros(ops.n, np.uint8)
        owned_rows[rows[np.flatnonzero(plan.owned)]] = 1
        self.owned = torch.as_tensor(owned_rows, device=dev)
        self.send = {s: torch.as_tensor(rows[i].astype(np.int32), device=dev)
                     for s, i in sorted(plan.send.items())}
        self.recv = {s: torch.as_tensor(rows[i].astype(np.int32), device=dev)
                     for s, i in sorted(plan.recv.items())}
        self.staged = dist.is_initialized() and dist.get_backend(group) == "gloo" and \
            torch.device(dev).type == "cuda"

    def _allreduce(self, values):
        t = self.torch.as_tensor(np.asarray(values, np.float64))
        if self.dist.is_initialized() and self.dist.get_world_size(self.group) > 1:
            if self.dist.get_backend(self.group) == "nccl":
                t = t.to(self.ops.device)
            self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def exchange(self, v):
        """Ghost rows of v <- their owners' values (one round of point-to-point
        messages with every neighbour, posted in rank order)."""
        torch, dist = self.torch, self.dist
        if not self.send and not self.recv:
            return 0
        bufs_out, bufs_in, ops = {}, {}, []
        for s, idx in self.send.items():
            b = torch.empty(idx.numel(), dtype=torch.float64, device=self.ops.device)
            self.ops.gather(idx, v, b)
            bufs_out[s] = b.cpu() if self.staged else b
        for s, idx in self.recv.items():
            bufs_in[s] = torch.empty(idx.numel(), dtype=torch.float64,
                                     device="cpu" if self.staged else self.ops.device)
        self.ops.synchronize()
        for peer in sorted(set(self.send) | set(self.recv)):
            if peer in self.send:
                ops.append(dist.P2POp(dist.isend, bufs_out[peer], peer, self.group))
            if peer in self.recv:
                ops.append(dist.P2POp(dist.irecv, bufs_in[peer], peer, self.group))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        moved = 0
        for s, idx in self.recv.items():
            b = bufs_in[s].to(self.ops.device) if self.staged else bufs_in[s]
            self.ops.scatter(idx, b, v)
            moved += idx.numel()
        return moved

    def solve(self, tol=1e-10, max_iterations=100000, relative=True, x0=None,
              variant="reference") -> ShardStats:
        """Solve the assembled system (ops.assemble first).  Returns the stats;
        the rank's owned solution rows are in self.x (SELL order).

        variant "reference": the reference's Jacobi-PCG recurrences
        (advanced_solvers.f90:880-925), two all-reduces and one halo exchange
        of p per iteration.  "single_reduction": the Chronopoulos-Gear form of
        the same method, whose (r, z), (A z, z) and (r, r) travel in ONE
        all-reduce of three doubles per iteration, with q = A p carried by
        recurrence and one halo exchange of z; it stops on the same
        recursive-residual rule, with rounding of a different order."""
        if variant == "single_reduction":
            return self._solve_single_reduction(tol, max_iterations, relative, x0)
        if variant != "reference":
            raise ValueError(f"unknown variant {variant!r}")
        ops, owned = self.ops, self.owned
        n = ops.n
        x = ops.zeros(n) if x0 is None else x0
        r, z, p, q = ops.zeros(n), ops.zeros(n), ops.zeros(n), ops.zeros(n)
        st = ShardStats()
        self.exchange(x)
        ops.spmv(x, q)
        rr, rz, bb = self._allreduce(ops.start(owned, q, r, z, p))
        st.allreduces += 1
        st.exchanged_values += self.exchange(p)
        r0 = np.sqrt(rr)
        st.initial_residual = r0
        target = tol * r0 if relative else tol
        res = r0
        if res <= target:
            st.converged = True
        it = 0
        while not st.converged and it < max_iterations:
            ops.spmv(p, q)
            (pq,) = self._allreduce([ops.dot(owned, p, q)])
            st.allreduces += 1
            if abs(pq) < 1.0e-14:   # the reference's breakdown test
                break
            alpha = rz / pq
            rr, rz_new = self._allreduce(ops.update(owned, alpha, p, q, x, r, z))
            st.allreduces += 1
            it += 1
            res = np.sqrt(rr)
            if res <= target:
                st.converged = True
                break
            beta = rz_new / rz
            rz = rz_new
            ops.direction(owned, beta, z, p)
            st.exchanged_values += self.exchange(p)
        st.iterations = it
        st.final_residual = float(res)
        self.x = x
        return st

    def _solve_single_reduction(self, tol, max_iterations, relative, x0) -> ShardStats:
        ops, owned = self.ops, self.owned
        n = ops.n
        x = ops.zeros(n) if x0 is None else x0
        r, z, p, s, w = ops.zeros(n), ops.zeros(n), ops.zeros(n), ops.zeros(n), ops.zeros(n)
        st = ShardStats()
        self.exchange(x)
        ops.spmv(x, w)
        ops.start(owned, w, r, z, p)          # r = b - A x, z = D^-1 r (its dots are not needed)
        st.exchanged_values += self.exchange(z)
        ops.spmv(z, w)
        gamma_old = alpha_old = 0.0
        target = None
        it = 0
        res = 0.0
        p.zero_()
        while True:
            gamma, delta, rr = self._allreduce(ops.cgs_dots(owned, r, z, w))
            st.allreduces += 1
            res = float(np.sqrt(rr))
            if target is None:
                st.initial_residual = res
                target = tol * res if relative else tol
            if res <= target:
                st.converged = True
                break
            if it >= max_iterations:
                break
            beta = gamma / gamma_old if it > 0 else 0.0
            denom = delta - (beta * gamma / alpha_old if it > 0 else 0.0)   # p^T A p
            if abs(denom) < 1.0e-14:   # the reference's breakdown test
                break
            alpha = gamma / denom
            ops.cgs_update(owned, alpha, beta, w, p, s, x, r, z)
            it += 1
            st.exchanged_values += self.exchange(z)
            ops.spmv(z, w)
            gamma_old, alpha_old = gamma, alpha
        st.iterations = it
        st.final_residual = res
        self.x = x
        return st

    def owned_solution(self):
        """(global free indices, values) of this rank's owned rows."""
        rows = self.ops.row_of_free[np.flatnonzero(self.plan.owned)]
        vals = self.x.cpu().numpy()[rows]
        return self.plan.sub_to_global_free[np.flatnonzero(self.plan.owned)], vals


def local_inputs(plan: RankPlan, vertices, cell_a=None, cell_b=None, samples=None,
                 constrained_values=None):
    """The rank's slices of global inputs: submesh vertices, per-cell arrays
    (cell-major, any trailing shape) and per-DoF constrained values."""
    v = np.asarray(vertices, float).reshape(-1, 3)[plan.vertex_ids]
    cut = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a)[plan.cells])
    g = None if constrained_values is None else \
        np.ascontiguousarray(np.asarray(constrained_values, float)[plan.sub_to_global_dof])
    return v, cut(cell_a), cut(cell_b), cut(samples), g


def solve_sharded(family: int, degree: int, vertices, cells, coef_a=1.0, coef_b=0.0,
                  cell_a=None, cell_b=None, samples=None, constrained_values=None,
                  boundary="all", rule=K.FFG_RULE_DUFFY, quadrature_degree=0, tol=1e-10,
                  max_iterations=100000, device=None, group=None, plans=None,
                  variant="reference"):
    """Solve one system over the ranks of the process group (one GPU each):
    returns (full solution on every rank, ShardStats).  samples is the
    cell-major array of source samples at the problem's sample points, as
    ffg_problem_solve takes it."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    if plans is None:
        plans = build_plans(family, degree, vertices, cells, world, boundary)
    plan = plans[rank]
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    ops = DeviceOps(plan, family, degree, rule, quadrature_degree, dev)
    try:
        v, ca, cb, smp, g = local_inputs(plan, vertices, cell_a, cell_b, samples,
                                         constrained_values)
        ops.assemble(v, coef_a, coef_b, ca, cb, smp, g)
        solver = ShardedSolver(plan, ops, group)
        st = solver.solve(tol=tol, max_iterations=max_iterations, variant=variant)
        full = gather_solution(solver, plan.n_dofs, plan.free_dofs, constrained_values)
        return full, st
    finally:
        ops.close()


def gather_solution(solver: ShardedSolver, n_dofs: int, free_dofs: np.ndarray,
                    constrained_values=None) -> np.ndarray:
    """The full solution (all DoFs) on every rank: owned rows all-gathered,
    constrained DoFs from constrained_values (or zero)."""
    import torch.distributed as dist
    idx, vals = solver.owned_solution()
    parts = [(idx, vals)]
    if dist.is_initialized() and dist.get_world_size(solver.group) > 1:
        parts = [None] * dist.get_world_size(solver.group)
        dist.all_gather_object(parts, (idx, vals), group=solver.group)
    full = np.zeros(n_dofs) if constrained_values is None else \
        np.where(np.isin(np.arange(n_dofs), free_dofs), 0.0, np.asarray(constrained_values, float))
    for i, v in parts:
        full[free_dofs[i]] = v
    return full
