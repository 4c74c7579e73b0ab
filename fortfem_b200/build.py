"""Build libfortfem_gpu.so in-tree for sm_100a with nvcc.

    python -m fortfem_b200.build            # incremental
    python -m fortfem_b200.build --force    # rebuild everything

Objects go to fortfem_b200/_build/; the shared library to
fortfem_b200/libfortfem_gpu.so.  The Nedelec tables include file is
regenerated first when it is missing.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfortfem_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-O3",
          "-I" + os.path.join(HERE, "..", "include")]
SOURCES = ["topology.cpp", "basis.cpp", "kernels_assemble.cu", "kernels_pcg.cu", "capi.cu",
           "noalloc.cu", "topology_gpu.cu", "kernels_ad.cu",
           "kernels_probe.cu", "kernels_pml.cu",
           "kernels_dist.cu", "kernels_weighted.cu", "kernels_tc.cu", "kernels_oriented.cu"]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".inc"))] + \
        [os.path.join(HERE, "..", "include", "fortfem_gpu.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    tables = os.path.join(CSRC, "nedelec_tables.inc")
    if not os.path.exists(tables):
        from fortfem_b200.gen_nedelec_tables import emit
        emit(tables)
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs, jobs = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            lang = ["-x", "cu"] if src.endswith(".cu") else []
            cmd = [NVCC, *ARCH, *COMMON, *lang, "-c", path, "-o", obj]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with ThreadPoolExecutor(max_workers=min(8, len(jobs) or 1)) as ex:
        for out in ex.map(run, jobs):
            if verbose and out:
                print(out, file=sys.stderr)
    if force or jobs or _stale(LIB, objs):
        run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lgomp"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
