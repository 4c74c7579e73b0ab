"""One system sharded over several ranks, on the CPU with gloo: the plan
(ownership, ghost layer, exchange lists) and the row-block Jacobi-PCG loop
with its halo exchange, against the single-system solve.  The ranks'
arithmetic runs on numpy (tests/shard_worker.py); the GPU kernels of the same
loop are covered by tests/test_gpu_sharding.py."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import oracle
from fortfem_b200 import _capi as K
from fortfem_b200 import sharding, synth

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(args, world, tmp_path, timeout=120, extra=()):
    port = _free_port()
    procs, outs = [], []
    for rank in range(world):
        out = tmp_path / f"shard_{rank}.json"
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"),
                                       *map(str, args), str(out), *extra], env=env))
        outs.append(out)
    codes = []
    for p in procs:
        try:
            codes.append(p.wait(timeout=timeout))
        except subprocess.TimeoutExpired:
            p.kill()
            codes.append(None)
    return codes, [json.loads(o.read_text()) if o.exists() else None for o in outs]


@pytest.mark.parametrize("world", [2, 3, 4])
def test_partition_is_deterministic_and_balanced(world):
    v, t = oracle.box_mesh([6, 6, 6])
    a = sharding.partition_cells(v, t, world)
    assert np.array_equal(a, sharding.partition_cells(v, t, world))
    counts = np.bincount(a, minlength=world)
    assert counts.min() > 0 and counts.max() - counts.min() <= 1


@pytest.mark.parametrize("family,degree", [(K.FFG_TETRA_LAGRANGE, 1), (K.FFG_TETRA_LAGRANGE, 3),
                                           (K.FFG_TETRA_NEDELEC, 2)])
@pytest.mark.parametrize("world", [2, 3])
def test_plans_cover_every_row_once_with_complete_rows(family, degree, world):
    v, t = oracle.box_mesh([4, 4, 3])
    v = synth.jitter_interior(v, 0.25, 0.1, 2)
    plans = sharding.build_plans(family, degree, v, t, world)
    topo = sharding.build_topology(family, degree, t, len(v), "all")
    gd, con = topo["global_dofs"], topo["constrained"]
    n_free = int((~con).sum())
    owned = np.concatenate([p.sub_to_global_free[p.owned] for p in plans])
    assert np.array_equal(np.sort(owned), np.arange(n_free))       # each row once
    free_index = np.full(topo["n_dofs"], -1)
    free_index[np.flatnonzero(~con)] = np.arange(n_free)
    for p in plans:
        # every cell that touches an owned row is assembled by its owner
        mine = set(p.sub_to_global_free[p.owned].tolist())
        touching = [c for c in range(len(t)) if mine & set(free_index[gd[c]].tolist())]
        assert set(p.cells.tolist()) == set(touching)
        # the submesh DoF map agrees with the global one, constrained flags too
        assert np.array_equal(p.constrained.astype(bool), con[p.sub_to_global_dof])
        # every ghost row is received exactly once, from its owner
        ghosts = np.flatnonzero(~p.owned)
        got = np.sort(np.concatenate([r for r in p.recv.values()])) if p.recv else np.array([])
        assert np.array_equal(got, ghosts)
        for s, rows in p.recv.items():
            q = plans[s]
            assert np.array_equal(q.sub_to_global_free[q.send[p.rank]], p.sub_to_global_free[rows])
            assert q.owned[q.send[p.rank]].all()


@pytest.mark.parametrize("family,degree,n", [(K.FFG_TETRA_LAGRANGE, 2, 4),
                                             (K.FFG_TETRA_NEDELEC, 1, 3)])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_pcg_matches_the_single_system(family, degree, n, world, tmp_path):
    codes, res = _run([family, degree, n], world, tmp_path)
    assert codes == [0] * world
    # the reference's rule (including its absolute |p^T A p| < 1e-14 stop) is
    # applied identically on every rank and by the single-system PCG
    assert {r["converged"] for r in res} == {res[0]["serial_converged"]}
    its = {r["iterations"] for r in res}
    assert len(its) == 1                      # every rank took the same decisions
    assert sum(r["owned"] for r in res) == res[0]["n_free"]
    # the same iterates as the single-system PCG up to the summation order of
    # the dot products
    assert abs(res[0]["iterations"] - res[0]["serial_iterations"]) <= 1
    assert res[0]["error"] < 1e-9
    assert all(r["exchanged"] > 0 for r in res)


@pytest.mark.parametrize("family,degree,n", [(K.FFG_TETRA_LAGRANGE, 2, 4),
                                             (K.FFG_TETRA_NEDELEC, 1, 3)])
@pytest.mark.parametrize("world", [2, 3])
def test_single_reduction_pcg_one_allreduce_per_iteration(family, degree, n, world, tmp_path):
    """The Chronopoulos-Gear form: one all-reduce per iteration (plus the final
    convergence check), the same stopping rule, the single-system solution."""
    codes, res = _run([family, degree, n], world, tmp_path, extra=("single_reduction",))
    assert codes == [0] * world
    its = {r["iterations"] for r in res}
    assert len(its) == 1
    it = res[0]["iterations"]
    assert all(r["allreduces"] == it + 1 for r in res)
    assert {r["converged"] for r in res} == {res[0]["serial_converged"]}
    assert abs(it - res[0]["serial_iterations"]) <= 2
    assert res[0]["error"] < 1e-8
