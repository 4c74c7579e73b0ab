"""Batched solves and the serving loop on the GPU.

A system solved in a batch must give the same bits as the same system solved
alone in its mode (one thread block per system, or the whole device): no
reduction crosses systems.  Against the synchronous cooperative path
(Problem.solve_device) solutions agree within 1e-6 of their largest entry;
both stop at true relative residual 1e-10 on systems whose condition number
stays below 1e4.
"""
import numpy as np
import pytest
import torch

from fortfem_b200 import serving as S

pytestmark = pytest.mark.gpu


def _run(eng, mode, reqs):
    tok = eng.launch(S.Batch(mode, reqs, 0))
    torch.cuda.synchronize()
    assert eng.done(tok)
    return eng.collect(tok)


def test_batch_matches_alone_and_the_cooperative_path():
    eng = S.DeviceEngine(keep_solutions=True)
    reqs = [S.Request(0, "p1", 12, 101), S.Request(1, "p2", 4, 102), S.Request(2, "p1", 40, 103),
            S.Request(3, "p2", 7, 104), S.Request(4, "p1", 25, 105)]
    for r in reqs:
        assert eng.can_host(r.key)
    mixed = _run(eng, "cta_per_system", reqs)
    for r, m in zip(reqs, mixed):
        assert m.converged and m.true_relative_residual <= 1e-10
        alone = _run(eng, "cta_per_system", [r])[0]
        assert np.array_equal(alone.solution, m.solution)
        whole = _run(eng, "whole_device", [r])[0]
        assert whole.converged and whole.true_relative_residual <= 1e-10
        mesh = eng.meshes[r.key][0]
        v, kappa, src = eng._inputs(mesh, r)
        ref = torch.empty(mesh.problem.n_dofs, dtype=torch.float64, device=eng.device)
        st = mesh.problem.solve_device(v, ref, 1.0, 0.0, kappa, None, src, None, eng.options)
        assert st.converged
        ref = ref.cpu().numpy()
        scale = np.abs(ref).max()
        assert scale > 0
        assert np.abs(m.solution - ref).max() <= 1e-6 * scale
        assert np.abs(whole.solution - ref).max() <= 1e-6 * scale
    eng.close()


def test_group_batch_matches_alone_and_the_whole_device():
    """Large systems side by side in one cooperative launch (FFG_BATCH_CTA_GROUPS),
    each on its own group of 2 to 22 thread blocks: the same bits as the system
    alone in a group launch, and within 1e-6 of the whole-device solve."""
    eng = S.DeviceEngine(keep_solutions=True)
    reqs = [S.Request(0, "p1", 200, 201), S.Request(1, "p2", 12, 202),
            S.Request(2, "p1", 600, 203), S.Request(3, "p1", 120, 204)]
    for r in reqs:
        assert eng.can_host(r.key)
    mixed = _run(eng, "cta_groups", reqs)
    for r, m in zip(reqs, mixed):
        assert m.converged and m.true_relative_residual <= 1e-10
        alone = _run(eng, "cta_groups", [r])[0]
        assert np.array_equal(alone.solution, m.solution)
        whole = _run(eng, "whole_device", [r])[0]
        assert whole.converged
        scale = np.abs(whole.solution).max()
        assert scale > 0 and np.abs(m.solution - whole.solution).max() <= 1e-6 * scale
    eng.close()


def test_one_block_system_with_more_than_32_slices_per_warp():
    # 18^3 x 6 P2: 42,875 free rows, 1,340 slices, so each of the block's 32
    # warps walks about 42 slices (past the 32 a warp keeps in registers)
    eng = S.DeviceEngine(keep_solutions=True)
    r = S.Request(0, "p2", 18, 211)
    assert eng.can_host(r.key)
    mesh = eng.meshes[r.key][0]
    assert mesh.problem.n_free > 32 * 32 * 32
    one = _run(eng, "cta_per_system", [r])[0]
    assert one.converged and one.true_relative_residual <= 1e-10
    v, kappa, src = eng._inputs(mesh, r)
    ref = torch.empty(mesh.problem.n_dofs, dtype=torch.float64, device=eng.device)
    st = mesh.problem.solve_device(v, ref, 1.0, 0.0, kappa, None, src, None, eng.options)
    assert st.converged
    ref = ref.cpu().numpy()
    assert np.abs(one.solution - ref).max() <= 1e-6 * np.abs(ref).max()
    eng.close()


def test_serving_stream_results_same_alone_and_in_the_mix():
    reqs = S.poisson_stream(40, 2000.0, seed=11, p1_range=(8, 96), p2_range=(4, 14))
    eng = S.DeviceEngine(keep_solutions=True)
    eng.prepare(reqs)
    sch = S.Scheduler(small_rows=2000, max_batch=16, streams=2)
    res = S.serve(reqs, eng, sch)
    assert [r.rid for r in res] == list(range(40))
    assert all(r.converged and r.true_relative_residual <= 1e-10 for r in res)
    assert any(r.batch_size > 1 for r in res)            # requests did share batches
    assert any(r.mode == "whole_device" for r in res)
    lat = S.percentiles([r.latency for r in res])
    assert 0 < lat["p50"] <= lat["p99"] <= lat["p99.9"]
    for r, got in zip(reqs, res):
        mode = "cta_per_system" if sch.is_small(r) else "whole_device"
        alone = _run(eng, mode, [r])[0]
        assert np.array_equal(alone.solution, got.solution)
    eng.close()


def test_same_size_requests_share_a_batch_and_overlap():
    """Three requests of one mesh size in one batch (three pool members), and
    a fourth in a batch on the other stream while the first is in flight:
    every result is the bits it gets alone."""
    eng = S.DeviceEngine(keep_solutions=True)
    reqs = [S.Request(i, "p2", 6, 300 + i) for i in range(3)] + [S.Request(3, "p1", 30, 400)]
    assert eng.can_host(("p2", 6), 4) and eng.can_host(("p1", 30), 1)
    assert len(eng.meshes[("p2", 6)]) == 4
    t1 = eng.launch(S.Batch("cta_per_system", reqs[:3], 0))
    t2 = eng.launch(S.Batch("cta_per_system", [reqs[3], S.Request(4, "p2", 6, 500)], 1))
    torch.cuda.synchronize()
    got = eng.collect(t1) + eng.collect(t2)
    assert all(g.converged and g.true_relative_residual <= 1e-10 for g in got)
    for r, g in zip(reqs + [S.Request(4, "p2", 6, 500)], got):
        alone = _run(eng, "cta_per_system", [r])[0]
        assert np.array_equal(alone.solution, g.solution)
    # different seeds on one mesh size give different systems
    assert not np.array_equal(got[0].solution, got[1].solution)
    eng.close()
