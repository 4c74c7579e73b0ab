"""Seeded synthetic inputs of the five workloads this path is measured on.

No public dataset is involved: meshes are the reference's own structured
generators, perturbed and decorated with seeded coefficients and sources.

* P1 unit square: ``unit_square_mesh(65)`` (64x64 squares, 8192 triangles,
  4225 nodes), coefficient 1, f = 1, homogeneous Dirichlet.
* P2 tetrahedra: 48^3 Kuhn box (663,552 cells, 912,673 DoFs), interior vertices
  jittered uniformly in [-0.1h, 0.1h]^3 (seed 2), per-cell coefficient
  exp(N(0,1)), source sin(pi x) sin(pi y) sin(pi z) sampled at the 4-point
  degree-two rule, homogeneous Dirichlet.
* Nedelec slabs: 24^3 Kuhn box, curl mu^-1 curl + kappa I with mu^-1 = 1 /
  1000 / 1 on z in [0,1/3) / [1/3,2/3) / [2/3,1] (by cell centroid), kappa = 1,
  J = (0,0,1) in the central slab, zero tangential trace on the boundary.
* Serving stream: Poisson arrivals of P1 and P2 Poisson requests with
  log-uniform sizes, lognormal cell coefficients and random-Fourier-feature
  Gaussian random field sources.
* Nedelec order 6 stress case: 12^3 Kuhn box jittered +-0.05h (seed 5),
  mu^-1 ~ U[0.5, 2], kappa = 10, smooth random trig source.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import api
from ._capi import FFG_RULE_DEGREE_TWO, FFG_RULE_DUFFY


def box_mesh(n: int):
    v, t, st = api.generate_structured_tetra_box_mesh([[0, 1], [0, 1], [0, 1]], [n, n, n])
    if st.code:
        raise api.FortfemError(st.code, "box mesh")
    return v, t


def jitter_interior(vertices: np.ndarray, h: float, delta: float, seed: int) -> np.ndarray:
    """Uniform jitter in [-delta h, delta h]^3 on vertices off the unit-cube boundary."""
    rng = np.random.default_rng(seed)
    v = vertices.copy()
    interior = np.all((v > 1e-12) & (v < 1 - 1e-12), axis=1)
    v[interior] += rng.uniform(-delta * h, delta * h, size=(int(interior.sum()), 3))
    return v


def jitter_interior_2d(vertices: np.ndarray, h: float, delta: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = vertices.copy()
    interior = np.all((v > 1e-12) & (v < 1 - 1e-12), axis=1)
    v[interior] += rng.uniform(-delta * h, delta * h, size=(int(interior.sum()), 2))
    return v


@dataclass
class ScalarCase:
    name: str
    family: int
    degree: int
    vertices: np.ndarray
    cells: np.ndarray
    rule: int
    quadrature_degree: int
    cell_coefficient: Optional[np.ndarray]
    source: object  # callable f(x, y, z) or None
    meta: dict = field(default_factory=dict)


def p2_poisson_case(n: int = 48, delta: float = 0.1, seed: int = 2, mesh=None) -> ScalarCase:
    """P2 tetrahedral Lagrange Poisson on n^3 x 6 jittered tets, lognormal coefficient.
    `mesh(n) -> (vertices, cells)` replaces the library's Kuhn box generator
    (a CPU-only caller passes a restatement of the same generator)."""
    v, t = (mesh or box_mesh)(n)
    v = jitter_interior(v, 1.0 / n, delta, seed)
    rng = np.random.default_rng(seed + 1000)
    kappa = np.exp(rng.standard_normal(len(t)))
    src = lambda x, y, z: np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)  # noqa: E731
    return ScalarCase("p2_tetra_poisson", 1, 2, v, t, FFG_RULE_DEGREE_TWO, 0, kappa, src,
                      dict(n=n, delta=delta, seed=seed))


def p1_square_case(n_vertices: int = 65) -> ScalarCase:
    v, t = api.unit_square_mesh(n_vertices)
    return ScalarCase("p1_unit_square", 3, 1, v, t, FFG_RULE_DUFFY, 0, None, None,
                      dict(n_vertices=n_vertices))


def slab_reluctivity(vertices: np.ndarray, cells: np.ndarray, values=(1.0, 1000.0, 1.0)) -> np.ndarray:
    zc = vertices[cells].mean(axis=1)[:, 2]
    return np.where(zc < 1.0 / 3.0, values[0], np.where(zc < 2.0 / 3.0, values[1], values[2]))


def slab_current(points: np.ndarray) -> np.ndarray:
    """J = (0, 0, 1) for 1/3 <= z < 2/3, else 0, at (..., 3) points."""
    z = points[..., 2]
    j = np.zeros(points.shape)
    j[..., 2] = np.where((z >= 1.0 / 3.0) & (z < 2.0 / 3.0), 1.0, 0.0)
    return j


def trig_vector_source(seed: int, modes: int = 8):
    """A smooth random vector field: sum of <= `modes` low-degree trig modes."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 3, size=(modes, 3))
    a = rng.standard_normal((modes, 3))
    ph = rng.uniform(0, 2 * np.pi, size=(modes,))

    def f(points):
        arg = np.pi * (points[..., None, :] * k).sum(-1) + ph
        return np.einsum("...m,mc->...c", np.cos(arg), a)
    return f


def grf_source(seed: int, correlation_length: float = 0.1, features: int = 64, dim: int = 3):
    """Gaussian random field by seeded random Fourier features, Gaussian spectrum."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((features, dim)) / correlation_length
    b = rng.uniform(0, 2 * np.pi, size=features)
    amp = np.sqrt(2.0 / features)

    def f(points):
        return amp * np.cos(points[..., :dim] @ w.T + b).sum(-1)
    return f


@dataclass
class CurlCase:
    """A curl mu^-1 curl + kappa I problem with zero tangential trace."""
    name: str
    order: int
    vertices: np.ndarray
    cells: np.ndarray
    cell_curl: np.ndarray      # mu^-1 per cell
    mass: float                # kappa
    source: object             # f(points (..., 3)) -> (..., 3)
    meta: dict = field(default_factory=dict)


def nedelec_slab_case(order: int, n: int = 24, mesh=None) -> CurlCase:
    """Three material slabs along z on an n^3 x 6 Kuhn box (no jitter):
    mu^-1 = 1 / 1000 / 1 by cell centroid, kappa = 1, J = (0, 0, 1) in the
    central slab."""
    v, t = (mesh or box_mesh)(n)
    return CurlCase("nedelec_slabs", order, v, t, slab_reluctivity(v, t), 1.0, slab_current,
                    dict(n=n))


def nedelec_order6_case(n: int = 12, delta: float = 0.05, seed: int = 5, mesh=None,
                        order: int = 6) -> CurlCase:
    """Order-6 stress case: n^3 x 6 Kuhn box jittered +-0.05h, mu^-1 ~ U[0.5, 2]
    per cell, kappa = 10, a smooth random trig vector source."""
    v, t = (mesh or box_mesh)(n)
    v = jitter_interior(v, 1.0 / n, delta, seed)
    rng = np.random.default_rng(seed + 1000)
    mu = rng.uniform(0.5, 2.0, len(t))
    return CurlCase("nedelec_order6", order, v, t, mu, 10.0, trig_vector_source(seed),
                    dict(n=n, delta=delta, seed=seed))
