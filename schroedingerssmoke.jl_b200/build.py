"""Build libisf.so (the sm_100a kernels + C ABI) in-tree with nvcc.

    python schroedingerssmoke.jl_b200/build.py [--force]

Each .cu under csrc/ is compiled in parallel to an object under _build/ and
linked into schroedingerssmoke.jl_b200/libisf.so.  Rebuilds only what is
older than its sources.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.environ.get("ISF_CSRC") or os.path.join(HERE, "csrc")
# ISF_CHECK=1 builds the bounds-checking debug variant libisf_check.so
CHECK = os.environ.get("ISF_CHECK", "0") == "1"
BUILD = os.environ.get("ISF_BUILD_DIR") or os.path.join(HERE, "_build_check" if CHECK else "_build")
LIB = os.environ.get("ISF_LIB_OUT") or os.path.join(HERE, "libisf_check.so" if CHECK else "libisf.so")
# extra nvcc flags, e.g. -DISF_ST_SZ=16 to build a tuning variant elsewhere
EXTRA = os.environ.get("ISF_EXTRA_FLAGS", "").split()
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", INCLUDE] + (["-DISF_CHECK"] if CHECK else []) + EXTRA


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, verbose):
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = _headers()
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            todo.append((s, o))
    logs = {}
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            futs = {ex.submit(_compile, s, o, verbose): s for s, o in todo}
            for f in cf.as_completed(futs):
                logs[futs[f]] = f.result()
    if force or todo or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    if verbose:
        for s, log in logs.items():
            print(f"== {os.path.basename(s)}\n{log}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
