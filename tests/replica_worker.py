"""One rank of the CPU (gloo) replica tests; run by tests/test_replicas_cpu.py.

Usage: python replica_worker.py <scenario> <out.json>  (RANK, WORLD_SIZE,
MASTER_ADDR, MASTER_PORT in the environment)."""
import datetime
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import torch.distributed as dist  # noqa: E402

from fortfem_b200 import replicas, serving  # noqa: E402


def main():
    scenario, out = sys.argv[1], sys.argv[2]
    rank, world, _ = replicas.env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=10))
    res = {"rank": rank}
    if scenario == "share":
        reqs = serving.poisson_stream(300, 100.0, seed=9)
        mine = replicas.partition_requests(reqs, world)[rank]
        res["mine"] = [r.rid for r in mine]
        res["all"] = replicas.gather_lists([r.rid for r in mine])
        res["max"] = replicas.max_over_ranks(float(rank + 1))
        res["sum"] = replicas.sum_over_ranks(float(sum(serving.free_dofs(r.key) for r in mine)))
        res["total"] = float(sum(serving.free_dofs(r.key) for r in reqs))
    elif scenario == "fail":
        # rank 1 fails between steps; rank 0 must learn of it from its next
        # collective instead of waiting for ever
        replicas.max_over_ranks(1.0)
        if rank == 1:
            os._exit(3)
        try:
            replicas.max_over_ranks(2.0)
            res["saw_failure"] = False
        except Exception as e:  # noqa: BLE001 - any collective error is the signal
            res["saw_failure"] = True
            res["error"] = type(e).__name__
    with open(out, "w") as f:
        json.dump(res, f)
    if scenario != "fail":
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
