"""The launch-shape autotuner (ffg_problem_autotune): it times candidate
shapes on the problem's own inputs, keeps the fastest, and the results of the
problem do not change beyond the PCG's partition-dependent rounding."""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu


def rel_frob(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("family,degree", [(K.FFG_TETRA_LAGRANGE, 2), (K.FFG_TETRA_NEDELEC, 2),
                                           (K.FFG_TETRA_NEDELEC, 3)])
def test_autotune_keeps_results_and_reports_times(family, degree):
    n = 8 if family == K.FFG_TETRA_LAGRANGE else 6
    v, t = oracle.box_mesh([n, n, n])
    v = synth.jitter_interior(v, 1.0 / n, 0.1, 3)
    kappa = np.exp(np.random.default_rng(degree).standard_normal(len(t)))
    with ff.Problem(family, degree, t, len(v), boundary="all") as prob:
        pts = prob.sample_points(v)
        if family == K.FFG_TETRA_NEDELEC:
            # a mass-dominated system, so that both solves reach the 1e-10 true residual
            src = synth.trig_vector_source(degree)(pts)
            cb = 50.0
        else:
            src = np.sin(np.pi * pts[..., 0]) * pts[..., 1]
            cb = 0.0
        R0, rhs0, _ = prob.reduced_system(v, 1.0, cb, kappa, None, src)
        sol0, st0 = prob.solve(v, 1.0, cb, kappa, None, src)
        tune = prob.autotune(v, 1.0, cb, kappa, None, src)
        print(tune)
        assert tune["assembly_ms"] > 0 and tune["assembly_ms"] <= tune["default_assembly_ms"]
        assert tune["solve_ms"] > 0 and tune["solve_ms"] <= tune["default_solve_ms"]
        assert tune["slice_cost"] in (16, 64, 128, 256, 512, 1024)
        if family == K.FFG_TETRA_NEDELEC:
            assert tune["element_threads"] in (0, 128, 256)
        R1, rhs1, _ = prob.reduced_system(v, 1.0, cb, kappa, None, src)
        sol1, st1 = prob.solve(v, 1.0, cb, kappa, None, src)
        # assembly is the same bits whatever the launch shape (same summation order)
        assert np.array_equal(R0.val, R1.val) and np.array_equal(rhs0, rhs1)
        assert st0.converged and st1.converged
        assert st1.true_relative_residual <= 1e-10
        assert np.linalg.norm(sol1 - sol0) <= 1e-6 * np.linalg.norm(sol0)
        # the choice applies to another problem of the same kind
        with ff.Problem(family, degree, t, len(v), boundary="all") as other:
            other.set_tuning(tune)
            R2, _, _ = other.reduced_system(v, 1.0, cb, kappa, None, src)
            assert np.array_equal(R2.val, R0.val)
        with pytest.raises(ff.FortfemError):
            prob.set_tuning({**tune, "element_threads": 100})
