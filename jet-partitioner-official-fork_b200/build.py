"""Builds libjetb200.so in-tree with nvcc for sm_100a.

    python jet-partitioner-official-fork_b200/build.py [--verbose-ptxas]

Each tier (int widths) is its own translation unit, compiled in parallel;
CUDA's bundled static Metis is linked in for the coarsest-graph partition.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libjetb200.so")
HELPER = os.path.join(HERE, "jet_metis_helper")
BUILD = os.path.join(HERE, "_build")
UNITS = ["runtime.cu", "tier_i32.cu", "tier_big.cu", "tier_biggest.cu", "noalloc.cu", "batch.cu", "metis_io.cpp", "test_hooks.cu"]
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
METIS = os.path.join(CUDA, "targets", "x86_64-linux", "lib", "libmetis_static.a")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp"))] + \
        [os.path.join(HERE, "..", "include", "jet_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT) or not os.path.exists(HELPER):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []

    def compile_unit(u):
        obj = os.path.join(BUILD, os.path.splitext(u)[0] + ".o")
        cmd = ["nvcc", *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, u), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return u, obj, r

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        results = list(ex.map(compile_unit, UNITS))
    objs = []
    for u, obj, r in results:
        if ptxas_verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s" % u)
        objs.append(obj)
    tmp = OUT + ".tmp"
    cmd = ["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs, METIS, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, OUT)
    # helper process for concurrent Metis calls (batched and served modes)
    cmd = ["g++", "-O2", "-o", HELPER + ".tmp", os.path.join(CSRC, "metis_helper.cpp"), METIS, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("metis helper build failed")
    os.replace(HELPER + ".tmp", HELPER)
    return OUT


if __name__ == "__main__":
    print(build(force=True, ptxas_verbose="--verbose-ptxas" in sys.argv))
