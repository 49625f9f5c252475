"""Builds libdq.so (the C-ABI library of include/dq.h) in-tree for sm_100a.

Every .cu file under dynaquant_b200/csrc is compiled with nvcc for
compute_100a/sm_100a, the C++ host under dynaquant_b200/host with g++, and
both are linked into dynaquant_b200/libdq.so; the command-line driver
dynaquant_b200/dq_propagate links against it.  Objects go
to dynaquant_b200/_build/.  Rebuilds only what changed (by mtime, headers
included).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
MAIN = "dq_propagate_main.cpp"
CLI = os.path.join(HERE, "dq_propagate")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdq.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE,
         "--expt-relaxed-constexpr"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def _compile_host(src: str) -> str:
    """The C++ host (input file, data files, run driver): g++, linked into the same library."""
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + glob.glob(os.path.join(HOST, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-I", INCLUDE, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hsrcs = sorted(s for s in glob.glob(os.path.join(HOST, "*.cpp")) if not s.endswith(MAIN))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs) + len(hsrcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs)) + list(ex.map(_compile_host, hsrcs))
    if not (os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs)):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    main_src = os.path.join(HOST, MAIN)
    if not (os.path.exists(CLI) and os.path.getmtime(CLI) >= max(os.path.getmtime(LIB), os.path.getmtime(main_src))):
        cmd = [CXX, "-O2", "-std=c++17", "-I", INCLUDE, main_src, "-o", CLI, "-L", HERE, "-ldq",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
