"""Several ranks on independent systems, on the CPU with gloo (world size 2):
the request split, the max / sum / gather bookkeeping, and a rank that fails
between steps being seen by the other rank."""
import json
import os
import socket
import subprocess
import sys

from fortfem_b200 import replicas, serving

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(scenario, world, tmp_path, timeout=60):
    port = _free_port()
    procs, outs = [], []
    for rank in range(world):
        out = tmp_path / f"{scenario}_{rank}.json"
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "replica_worker.py"),
                                       scenario, str(out)], env=env))
        outs.append(out)
    codes = []
    for p in procs:
        try:
            codes.append(p.wait(timeout=timeout))
        except subprocess.TimeoutExpired:
            p.kill()
            codes.append(None)
    return codes, [json.loads(o.read_text()) if o.exists() else None for o in outs]


def test_partition_is_deterministic_complete_and_balanced():
    reqs = serving.poisson_stream(1000, 50.0, seed=3)
    shares = replicas.partition_requests(reqs, 4)
    assert shares == replicas.partition_requests(reqs, 4)
    ids = sorted(r.rid for s in shares for r in s)
    assert ids == list(range(1000))
    loads = [sum(serving.free_dofs(r.key) for r in s) for s in shares]
    biggest = max(serving.free_dofs(r.key) for r in reqs)
    assert max(loads) - min(loads) <= biggest      # greedy least-loaded bound
    assert replicas.partition_requests(reqs, 1) == [sorted(reqs, key=lambda r: (r.arrival, r.rid))]


def test_two_gloo_ranks_share_the_stream_and_agree_on_totals(tmp_path):
    codes, res = _run("share", 2, tmp_path)
    assert codes == [0, 0]
    a, b = res
    assert set(a["mine"]).isdisjoint(b["mine"])
    assert sorted(a["mine"] + b["mine"]) == list(range(300))
    assert a["all"] == b["all"] == a["mine"] + b["mine"]
    assert a["max"] == b["max"] == 2.0
    assert a["sum"] == b["sum"] == a["total"]


def test_rank_failure_between_steps_is_seen_by_the_other_rank(tmp_path):
    codes, res = _run("fail", 2, tmp_path)
    assert codes[1] == 3
    assert codes[0] == 0 and res[0]["saw_failure"] is True
