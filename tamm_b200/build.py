"""Build recipe for libtamm_b200.so (sm_100a) — run by __graft_entry__.build().

Compiles every CUDA / C++ source in tamm_b200/csrc with nvcc for sm_100a only and
links one shared library in-tree (tamm_b200/libtamm_b200.so).  Objects are cached
under tamm_b200/_build/ and rebuilt when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtamm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", f"-I{INCLUDE}", f"-I{CSRC}"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _compile(src, verbose=False, extra=()):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + COMMON + list(extra) + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "cu"] + ARCH + list(extra) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, ptxas_info=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = _headers()
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    todo = [s for s in srcs if force or ptxas_info or
            _stale(os.path.join(BUILD, os.path.basename(s) + ".o"), s, deps)]
    logs = {}
    if todo:
        with ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for src, (obj, err) in zip(todo, ex.map(lambda s: _compile(s, verbose, extra), todo)):
                logs[src] = err
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcuda"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    if ptxas_info:
        for src, err in logs.items():
            print(f"== {os.path.basename(src)}\n{err}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv, force="-f" in sys.argv)
    print(LIB)
