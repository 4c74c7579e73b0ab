"""Test infrastructure, not product code: the FP64 floor of the true relative
residual ||b - A x|| / ||b|| of a constrained system assembled by the oracle.

The solution closest to the exact one that FP64 can hold is found by
iterative refinement of a sparse LU solve (SuperLU through scipy) with the
residual accumulated in 80-bit long double; its residual, again evaluated in
long double, is the smallest true residual any FP64 solver can report for
this system (up to the refinement's own convergence).  The script prints it
next to eps || |A| |x| || / ||b|| (the rounding of one FP64 evaluation of
b - A x) and the condition-number-free bound the Jacobi-PCG runs against.

    python oracle/residual_floor.py slab 24 1      # Nedelec slab system, order 1
    python oracle/residual_floor.py p2 48          # the P2 Poisson system
"""
import json
import os
import sys
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from fortfem_b200 import synth  # noqa: E402


def system(kind, n, k=1):
    mesh = lambda m: oracle.box_mesh([m, m, m])  # noqa: E731
    if kind == "slab":
        c = synth.nedelec_slab_case(k, n, mesh=mesh)
        N, cp, ri, val = oracle.nedelec_csc(c.vertices, c.cells, k, 1.0, c.mass, c.cell_curl)
        pts = oracle.nedelec_load_points(c.vertices, c.cells, k)
        rhs = oracle.nedelec_load_samples(c.vertices, c.cells, k, c.source(pts))
        con = oracle.pec_mask(k, c.cells)
    else:
        c = synth.p2_poisson_case(n, mesh=mesh)
        v, t = c.vertices, c.cells
        N, cp, ri, val = oracle.lagrange_csc(v, t, 2, 1, 0, 1.0, 0.0, c.cell_coefficient)
        pts = oracle.lagrange_quadrature_points(v, t, 1, 0)
        rhs = oracle.lagrange_load_samples(v, t, 2, c.source(pts[..., 0], pts[..., 1], pts[..., 2]),
                                           1, 0)
        con, _ = oracle.lagrange_dirichlet(2, v, t)
    nf, rcp, rri, rv, rr, free = oracle.reduce_constrained(N, cp, ri, val, rhs, con)
    return sp.csc_matrix((rv, rri, rcp), shape=(nf, nf)), rr


def floor(A, b, sweeps=5):
    Acsr = A.tocsr()
    rows = np.repeat(np.arange(A.shape[0]), np.diff(Acsr.indptr))
    data_ld = Acsr.data.astype(np.longdouble)

    def resid(x):
        ax = np.zeros(A.shape[0], np.longdouble)
        np.add.at(ax, rows, data_ld * x.astype(np.longdouble)[Acsr.indices])
        return b.astype(np.longdouble) - ax

    t0 = time.perf_counter()
    lu = sla.splu(A.tocsc(), permc_spec="MMD_AT_PLUS_A")
    t_lu = time.perf_counter() - t0
    bn = float(np.linalg.norm(b))
    x = lu.solve(b)
    hist = []
    for _ in range(sweeps):
        r = resid(x)
        hist.append(float(np.sqrt((r * r).sum())) / bn)
        x = (x.astype(np.longdouble) + lu.solve(np.asarray(r, np.float64))).astype(np.float64)
    r = resid(x)
    hist.append(float(np.sqrt((r * r).sum())) / bn)
    rounding = float(np.finfo(np.float64).eps * np.linalg.norm(abs(A) @ abs(x)) / bn)
    return dict(n=A.shape[0], nnz=int(A.nnz), factor_seconds=t_lu, refinement=hist,
                floor=min(hist), eval_rounding=rounding)


if __name__ == "__main__":
    kind, n = sys.argv[1], int(sys.argv[2])
    k = int(sys.argv[3]) if len(sys.argv) > 3 else 1
    A, b = system(kind, n, k)
    out = floor(A, b)
    out.update(kind=kind, n_cells_side=n, order=k)
    print(json.dumps(out))
