"""One rank of the GPU sharded-solve test: several ranks share one GPU and
exchange their halos through gloo (host memory), so no kernel waits on
another rank.  Run by tests/test_gpu_sharding.py.

Usage: python shard_gpu_worker.py <family> <degree> <n> <out.npz> [variant]  (RANK,
WORLD_SIZE, MASTER_ADDR, MASTER_PORT in the environment)."""
import datetime
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from fortfem_b200 import replicas, sharding  # noqa: E402
from shard_gpu_case import case  # noqa: E402


def main():
    family, degree, n, out = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
    variant = sys.argv[5] if len(sys.argv) > 5 else "reference"
    rank, world, _ = replicas.env()
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    c = case(family, degree, n)
    full, st = sharding.solve_sharded(family, degree, c["v"], c["t"], c["coef"][0], c["coef"][1],
                                      samples=c["samples"], constrained_values=c["g"],
                                      quadrature_degree=c["q"], tol=1e-10,
                                      device=torch.device("cuda", 0), variant=variant)
    np.savez(out, full=full, iterations=st.iterations, converged=st.converged,
             exchanged=st.exchanged_values, allreduces=st.allreduces)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
