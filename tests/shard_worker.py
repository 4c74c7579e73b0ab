"""One rank of the CPU (gloo) sharded-solve tests; run by tests/test_sharding_cpu.py.

The rank's arithmetic is done here with numpy on the oracle's assembly of the
rank's submesh (test infrastructure standing in for the GPU kernels); the
plan, the exchange, the all-reduces and the iteration are the product's
(fortfem_b200.sharding).

Usage: python shard_worker.py <family> <degree> <n> <out.json>  (RANK,
WORLD_SIZE, MASTER_ADDR, MASTER_PORT in the environment)."""
import datetime
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import oracle  # noqa: E402
from fortfem_b200 import _capi as K  # noqa: E402
from fortfem_b200 import replicas, sharding, synth  # noqa: E402


class NumpyOps:
    """The DeviceOps interface on the CPU: the submesh's constrained system
    from the oracle, rows in the submesh's free order."""

    def __init__(self, plan, family, degree, vertices, source, constrained_values, coef):
        self.device = "cpu"
        v = vertices[plan.vertex_ids]
        t = plan.sub_cells
        g = np.where(plan.constrained.astype(bool), constrained_values[plan.sub_to_global_dof], 0.0)
        if family == K.FFG_TETRA_LAGRANGE:
            q = 2 * degree + 4
            n, cp, ri, val = oracle.lagrange_csc(v, t, degree, 0, q, coef[0], coef[1])
            pts = oracle.lagrange_quadrature_points(v, t, 0, q)
            rhs = oracle.lagrange_load_samples(v, t, degree, source(pts), 0, q)
        else:
            n, cp, ri, val = oracle.nedelec_csc(v, t, degree, coef[0], coef[1])
            pts = oracle.nedelec_load_points(v, t, degree)
            rhs = oracle.nedelec_load_samples(v, t, degree, source(pts))
        nf, rcp, rri, rv, rr, free = oracle.reduce_constrained(n, cp, ri, val, rhs,
                                                               plan.constrained, g)
        self.A = oracle.csc_to_scipy(nf, rcp, rri, rv).tocsr()
        self.n = nf
        self.row_of_free = np.arange(nf)
        d = self.A.diagonal()
        self.dinv = np.where(np.abs(d) > 1e-14, 1.0 / np.where(d == 0, 1, d), 1.0)
        self.b = rr

    def zeros(self, n):
        return torch.zeros(max(n, 1), dtype=torch.float64)

    def spmv(self, x, y):
        y.numpy()[: self.n] = self.A @ x.numpy()[: self.n]

    def start(self, owned, ax, r, z, p):
        o = owned.numpy()[: self.n].astype(bool)
        rr_ = np.where(o, self.b - ax.numpy()[: self.n], r.numpy()[: self.n])
        r.numpy()[: self.n] = rr_
        z.numpy()[: self.n] = np.where(o, self.dinv * rr_, z.numpy()[: self.n])
        p.numpy()[: self.n] = np.where(o, z.numpy()[: self.n], p.numpy()[: self.n])
        rv, zv = r.numpy()[: self.n][o], z.numpy()[: self.n][o]
        return np.array([rv @ rv, rv @ zv, self.b[o] @ self.b[o]])

    def update(self, owned, alpha, p, q, x, r, z):
        o = owned.numpy()[: self.n].astype(bool)
        X, R, Z, Pp, Q = (a.numpy()[: self.n] for a in (x, r, z, p, q))
        X[o] += alpha * Pp[o]
        R[o] -= alpha * Q[o]
        Z[o] = self.dinv[o] * R[o]
        return np.array([R[o] @ R[o], R[o] @ Z[o]])

    def dot(self, owned, a, b):
        o = owned.numpy()[: self.n].astype(bool)
        return float(a.numpy()[: self.n][o] @ b.numpy()[: self.n][o])

    def cgs_dots(self, owned, r, z, w):
        o = owned.numpy()[: self.n].astype(bool)
        R, Z, W = (a.numpy()[: self.n][o] for a in (r, z, w))
        return np.array([R @ Z, W @ Z, R @ R])

    def cgs_update(self, owned, alpha, beta, w, p, s, x, r, z):
        o = owned.numpy()[: self.n].astype(bool)
        W, P, S, X, R, Z = (a.numpy()[: self.n] for a in (w, p, s, x, r, z))
        P[o] = Z[o] + beta * P[o]
        S[o] = W[o] + beta * S[o]
        X[o] += alpha * P[o]
        R[o] -= alpha * S[o]
        Z[o] = self.dinv[o] * R[o]

    def direction(self, owned, beta, z, p):
        o = owned.numpy()[: self.n].astype(bool)
        P, Z = p.numpy()[: self.n], z.numpy()[: self.n]
        P[o] = Z[o] + beta * P[o]

    def gather(self, idx, src, dst):
        dst.numpy()[:] = src.numpy()[idx.numpy()]

    def scatter(self, idx, src, dst):
        dst.numpy()[idx.numpy()] = src.numpy()

    def synchronize(self):
        pass


def main():
    family, degree, n, out = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
    variant = sys.argv[5] if len(sys.argv) > 5 else "reference"
    rank, world, _ = replicas.env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=30))
    v, t = oracle.box_mesh([n, n, n])
    v = synth.jitter_interior(v, 1.0 / n, 0.1, 5)
    if family == K.FFG_TETRA_LAGRANGE:
        source = lambda pts: np.sin(3 * pts[..., 0]) + pts[..., 1] * pts[..., 2]
        boundary = "all"
        coef = (1.0, 0.5)
    else:
        source = lambda pts: np.stack([np.sin(2 * pts[..., 1]), pts[..., 2], 1.0 + 0 * pts[..., 0]],
                                      -1)
        boundary = "all"
        coef = (1.0, 1.0)
    plans = sharding.build_plans(family, degree, v, t, world, boundary)
    plan = plans[rank]
    topo = sharding.build_topology(family, degree, t, len(v), boundary)
    nd = topo["n_dofs"]
    free = np.flatnonzero(~topo["constrained"])
    assert plan.n_dofs == nd and np.array_equal(plan.free_dofs, free)
    g = np.zeros(nd)
    if family == K.FFG_TETRA_LAGRANGE:
        # nonzero Dirichlet data on the boundary DoFs (values per DoF)
        g = np.cos(np.arange(nd) * 0.37)
    ops = NumpyOps(plan, family, degree, v, source, g, coef)
    solver = sharding.ShardedSolver(plan, ops)
    st = solver.solve(tol=1e-10, max_iterations=5000, variant=variant)
    full = sharding.gather_solution(solver, nd, free, g)
    res = {"rank": rank, "iterations": st.iterations, "converged": bool(st.converged),
           "owned": int(plan.owned.sum()), "exchanged": int(st.exchanged_values),
           "allreduces": int(st.allreduces)}
    if rank == 0:
        # the single-system solve of the same problem by the oracle
        if family == K.FFG_TETRA_LAGRANGE:
            q = 2 * degree + 4
            nn, cp, ri, val = oracle.lagrange_csc(v, t, degree, 0, q, coef[0], coef[1])
            pts = oracle.lagrange_quadrature_points(v, t, 0, q)
            rhs = oracle.lagrange_load_samples(v, t, degree, source(pts), 0, q)
        else:
            nn, cp, ri, val = oracle.nedelec_csc(v, t, degree, coef[0], coef[1])
            pts = oracle.nedelec_load_points(v, t, degree)
            rhs = oracle.nedelec_load_samples(v, t, degree, source(pts))
        con = topo["constrained"]
        nf, rcp, rri, rv, rr, fr = oracle.reduce_constrained(nn, cp, ri, val, rhs, con,
                                                             np.where(con, g, 0.0))
        # the oracle's restatement of the reference PCG (same stopping rule)
        xs, ps = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=1e-10, relative=True, jacobi=True)
        ref = np.where(con, g, 0.0)
        ref[fr] = xs
        res["error"] = float(np.abs(full - ref).max() / max(1.0, np.abs(ref).max()))
        res["serial_iterations"] = ps["iterations"]
        res["serial_converged"] = ps["converged"]
        res["n_free"] = int(nf)
    with open(out, "w") as f:
        json.dump(res, f)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
