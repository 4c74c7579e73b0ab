"""The shared problem of the GPU sharded-solve tests (Lagrange with nonzero
Dirichlet data, or Nedelec with PEC), its source samples and the oracle's
single-system PCG solution (the reference's algorithm on the CPU)."""
import numpy as np

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth


def case(family, degree, n):
    v, t = oracle.box_mesh([n, n, n])
    v = synth.jitter_interior(v, 1.0 / n, 0.1, 5)
    if family == K.FFG_TETRA_LAGRANGE:
        q = 2 * degree + 4
        with ff.Problem(family, degree, t, len(v), quadrature_degree=q, boundary="all") as P:
            pts = P.sample_points(v)
            nd = P.n_dofs
        samples = np.sin(3 * pts[..., 0]) + pts[..., 1] * pts[..., 2]
        g = np.cos(np.arange(nd) * 0.37)
        coef = (1.0, 0.5)
    else:
        q = 0
        with ff.Problem(family, degree, t, len(v), boundary="all") as P:
            pts = P.sample_points(v)
            nd = P.n_dofs
        samples = np.stack([np.sin(2 * pts[..., 1]), pts[..., 2], 1.0 + 0 * pts[..., 0]], -1)
        g = np.zeros(nd)
        coef = (1.0, 1.0)
    return dict(v=v, t=t, q=q, samples=samples, g=g, coef=coef, nd=nd)


def oracle_solution(family, degree, c, tol=1e-10):
    v, t = c["v"], c["t"]
    if family == K.FFG_TETRA_LAGRANGE:
        n, cp, ri, val = oracle.lagrange_csc(v, t, degree, 0, c["q"], *c["coef"])
        rhs = oracle.lagrange_load_samples(v, t, degree, c["samples"], 0, c["q"])
        con, _ = oracle.lagrange_dirichlet(degree, v, t)
    else:
        n, cp, ri, val = oracle.nedelec_csc(v, t, degree, *c["coef"])
        rhs = oracle.nedelec_load_samples(v, t, degree, c["samples"])
        con = oracle.pec_mask(degree, t)
    g = np.where(con, c["g"], 0.0)
    nf, rcp, rri, rv, rr, fr = oracle.reduce_constrained(n, cp, ri, val, rhs, con, g)
    xs, st = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=tol, relative=True, jacobi=True)
    full = g.copy()
    full[fr] = xs
    return full, st
