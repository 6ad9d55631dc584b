"""Builds the CUDA library rfmanta_b200/librfmanta_b200.so for sm_100a.

    python -m rfmanta_b200.build [--verbose]

Every .cu file under csrc/ is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into _build/, every
host-only .cc file there with g++ (IEEE float, no contraction), and all are
linked into one shared library next to this file, so it travels with the
source tree.  Host objects use the image's g++ through nvcc.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(os.path.dirname(HERE), "_build", "rfmanta_b200")
LIB = os.path.join(HERE, "librfmanta_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]
CXX = "/usr/bin/g++"
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off",
            "-fno-fast-math"]


def _deps(src: str) -> list[str]:
    return [src] + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h"))


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, _deps(s)) or ptxas_info:
            cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for s in sorted(glob.glob(os.path.join(CSRC, "*.cc"))):
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".host.o")
        objs.append(o)
        if _stale(o, _deps(s)):
            jobs.append([CXX, *CXXFLAGS, "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for err in ex.map(run, jobs):
            if err and (verbose or ptxas_info):
                print(err, file=sys.stderr)
    if jobs or not os.path.exists(LIB) or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-ccbin", "/usr/bin/g++",
               "-Xcompiler", "-fPIC"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
