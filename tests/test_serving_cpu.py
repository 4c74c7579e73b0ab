"""Serving loop logic without a GPU: request streams, batch formation and the
replay loop against a simulated engine."""
import numpy as np

from fortfem_b200 import serving as S
from fortfem_b200 import build_topology, unit_square_mesh
from fortfem_b200 import FFG_TETRA_LAGRANGE, FFG_TRIANGLE_P1
from fortfem_b200.synth import box_mesh


def test_poisson_stream_shape():
    reqs = S.poisson_stream(4096, 100.0, seed=4)
    assert reqs == S.poisson_stream(4096, 100.0, seed=4)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert abs(arr[-1] - 4096 / 100.0) < 4.0            # mean gap 1/rate
    p1 = [r.n for r in reqs if r.family == "p1"]
    p2 = [r.n for r in reqs if r.family == "p2"]
    assert abs(len(p1) / 4096 - 0.7) < 0.03
    assert min(p1) >= 32 and max(p1) <= 1024 and min(p2) >= 8 and max(p2) <= 40
    # log-uniform: the median sits near the geometric mean of the range
    assert abs(np.log(np.median(p1)) - 0.5 * np.log(32 * 1024)) < 0.15


def test_free_dofs_match_topology():
    for n in (3, 5):
        v, t = unit_square_mesh(n + 1)
        topo = build_topology(FFG_TRIANGLE_P1, 1, t, len(v), boundary="all")
        assert topo["n_free"] == S.free_dofs(("p1", n))
        v, t = box_mesh(n)
        topo = build_topology(FFG_TETRA_LAGRANGE, 2, t, len(v), boundary="all")
        assert topo["n_free"] == S.free_dofs(("p2", n))


def test_scheduler_batches_small_requests_fifo():
    sch = S.Scheduler(small_rows=1000, max_batch=3, streams=2)
    reqs = [S.Request(i, "p1", 10 + i, i) for i in range(5)]
    sch.queue.extend(reqs)
    b = sch.next_batch(lambda k, n: True)
    assert b.mode == "cta_per_system" and [r.rid for r in b.requests] == [0, 1, 2]
    sch.inflight.append(b)
    b2 = sch.next_batch(lambda k, n: True)
    assert [r.rid for r in b2.requests] == [3, 4] and b2.slot != b.slot
    sch.inflight.append(b2)
    assert sch.next_batch(lambda k, n: True) is None        # both stream slots busy


def test_scheduler_same_mesh_size_shares_batches_up_to_the_pool():
    reqs = [S.Request(0, "p1", 10, 1), S.Request(1, "p1", 10, 2), S.Request(2, "p1", 11, 3),
            S.Request(3, "p1", 10, 4)]
    # a pool of one problem per size: one request of a size at a time
    sch = S.Scheduler(small_rows=1000, max_batch=8, streams=2)
    sch.queue.extend(reqs)
    b = sch.next_batch(lambda k, n: n <= 1)
    assert [r.rid for r in b.requests] == [0, 2]
    sch.inflight.append(b)
    assert sch.next_batch(lambda k, n: n <= 1) is None   # size 10 still in flight
    # a pool of two: two of size 10 in the first batch, the third in the next
    sch = S.Scheduler(small_rows=1000, max_batch=8, streams=2)
    sch.queue.extend(reqs)
    b = sch.next_batch(lambda k, n: n <= 2)
    assert [r.rid for r in b.requests] == [0, 1, 2]
    sch.inflight.append(b)
    assert sch.next_batch(lambda k, n: n <= 2) is None
    sch.inflight.clear()
    assert [r.rid for r in sch.next_batch(lambda k, n: n <= 2).requests] == [3]


def test_scheduler_large_request_waits_for_drain_and_runs_alone():
    sch = S.Scheduler(small_rows=100, max_batch=8, streams=2)
    small = S.Request(0, "p1", 5, 1)
    large = S.Request(1, "p2", 20, 2)
    later = S.Request(2, "p1", 6, 3)
    sch.queue.extend([small, large, later])
    b = sch.next_batch(lambda k, n: True)
    assert [r.rid for r in b.requests] == [0]            # stops at the first large request
    sch.inflight.append(b)
    assert sch.next_batch(lambda k, n: True) is None        # the large one waits for the drain
    sch.inflight.clear()
    b = sch.next_batch(lambda k, n: True)
    assert b.mode == "whole_device" and [r.rid for r in b.requests] == [1]
    sch.inflight.append(b)
    assert sch.next_batch(lambda k, n: True) is None        # nothing runs beside it


def test_small_requests_pass_a_large_one_only_within_the_window():
    sch = S.Scheduler(small_rows=100, max_batch=8, streams=2, bypass_window=0.05)
    busy = S.Request(9, "p1", 4, 9, arrival=0.0)
    large = S.Request(1, "p2", 20, 2, arrival=1.00)
    small = S.Request(2, "p1", 6, 3, arrival=1.01)
    sch.inflight.append(S.Batch("cta_per_system", [busy], 0))
    sch.queue.extend([large, small])
    b = sch.next_batch(lambda k, n: True, now=1.02)      # the large one waited 20 ms
    assert b.mode == "cta_per_system" and [r.rid for r in b.requests] == [2]
    sch.queue.append(S.Request(3, "p1", 7, 4, arrival=1.07))
    assert sch.next_batch(lambda k, n: True, now=1.08) is None   # waited 80 ms: no more passing
    sch.inflight.clear()
    b = sch.next_batch(lambda k, n: True, now=1.09)
    assert b.mode == "whole_device" and [r.rid for r in b.requests] == [1]


def test_scheduler_groups_large_requests_that_fit_the_grid():
    # free DoFs: p1 n -> (n-1)^2; group_rows 100 -> blocks ceil(free / 100), 2 .. grid
    sch = S.Scheduler(small_rows=100, max_batch=8, streams=2, groups=True, grid=10,
                      group_rows=100, max_groups=3)
    assert sch.group_ctas(("p1", 12)) == 2            # 121 free DoFs
    assert sch.group_ctas(("p1", 31)) == 9            # 900
    assert sch.group_ctas(("p1", 60)) == 10           # capped at the grid
    reqs = [S.Request(0, "p1", 12, 1), S.Request(1, "p1", 5, 2), S.Request(2, "p1", 31, 3),
            S.Request(3, "p1", 16, 4), S.Request(4, "p1", 13, 5), S.Request(5, "p1", 14, 6)]
    sch.queue.extend(reqs)
    b = sch.next_batch(lambda k, n: True)
    # head (2 blocks) + 16 (3 blocks) + 13 (2 blocks): 31 (9) does not fit, the small one waits,
    # and max_groups stops the scan
    assert b.mode == "cta_groups" and [r.rid for r in b.requests] == [0, 3, 4]
    sch.inflight.append(b)
    assert sch.next_batch(lambda k, n: True) is None        # nothing runs beside a group launch
    sch.inflight.clear()
    b = sch.next_batch(lambda k, n: True)
    assert b.mode == "cta_per_system" and [r.rid for r in b.requests] == [1]


def test_scheduler_skips_sizes_the_engine_cannot_host():
    sch = S.Scheduler(small_rows=1000, max_batch=8, streams=1)
    sch.queue.extend([S.Request(0, "p1", 10, 1), S.Request(1, "p1", 12, 2)])
    b = sch.next_batch(lambda k, n: k[1] != 10)
    assert [r.rid for r in b.requests] == [1]
    assert [r.rid for r in sch.queue] == [0]


class FakeEngine:
    """Completes a batch after a simulated device time proportional to its work."""

    def __init__(self, clock):
        self.clock = clock
        self.launched = []

    def can_host(self, key, count=1):
        return True

    def launch(self, b):
        work = sum(S.free_dofs(r.key) for r in b.requests)
        self.launched.append(b)
        return (self.clock() + 1e-9 * work, b)

    def done(self, token):
        return self.clock() >= token[0]

    def collect(self, token):
        return [S.Result(r.rid, 0.0, True, 10, 1e-11, "", 0) for r in token[1].requests]


def test_serve_replays_every_request_once_with_latencies():
    reqs = S.poisson_stream(200, 2000.0, seed=7, p1_range=(8, 64), p2_range=(4, 12))
    t = [0.0]

    def clock():
        t[0] += 1e-5
        return t[0]

    eng = FakeEngine(clock)
    res = S.serve(reqs, eng, S.Scheduler(small_rows=2000, max_batch=16, streams=2), clock=clock,
                  idle_sleep=0.0)
    assert [r.rid for r in res] == list(range(200))
    assert all(r.latency > 0 for r in res)
    modes = {r.mode for r in res}
    assert modes <= {"cta_per_system", "whole_device"}
    # whole-device batches hold one request and run with nothing beside them
    for b in eng.launched:
        if b.mode == "whole_device":
            assert len(b.requests) == 1
    stats = S.percentiles([r.latency for r in res])
    assert stats["p50"] <= stats["p99"] <= stats["p99.9"]


class _Pool:
    """Stand-in for a device problem of one mesh size (memory only)."""

    class problem:
        @staticmethod
        def close():
            pass


def _engine_with_budget(budget, per_pool):
    # the engine's pool logic without a device: creation books `per_pool` bytes
    eng = object.__new__(S.DeviceEngine)
    eng.budget, eng.used = budget, 0
    eng.meshes, eng.idle, eng.bytes, eng.last_use = {}, {}, {}, {}
    eng.max_instances = 8
    eng.setup_seconds = 0.0

    def create(key):
        m = _Pool()
        eng.meshes.setdefault(key, []).append(m)
        eng.idle.setdefault(key, []).append(m)
        eng.bytes[key] = eng.bytes.get(key, 0) + per_pool
        eng.used += per_pool
        return m

    eng._create = create
    eng._estimate = lambda key: per_pool
    return eng


def test_evictions_spare_the_sizes_of_the_batch_being_formed():
    a, b, c = ("p1", 100), ("p1", 200), ("p1", 300)
    eng = _engine_with_budget(budget=2, per_pool=1)
    assert eng.can_host(a) and eng.can_host(b)
    eng.last_use = {a: 0.0, b: 1.0}           # a is the least recently used
    # hosting c for a batch that already holds a must evict b, not a
    assert eng.can_host(c, 1, keep=frozenset({a}))
    assert set(eng.meshes) == {a, c}
    # with both other sizes kept there is nothing to evict
    assert not eng.can_host(b, 1, keep=frozenset({a, c}))
    # growing a pool never evicts that pool itself
    eng2 = _engine_with_budget(budget=1, per_pool=1)
    assert eng2.can_host(a)
    assert not eng2.can_host(a, 2)
    assert len(eng2.meshes[a]) == 1
