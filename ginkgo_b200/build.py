"""Builds ginkgo_b200/libginkgo_b200.so from ginkgo_b200/csrc/*.cu with nvcc
for sm_100a only.  Objects go to ginkgo_b200/_build/; a source is recompiled
when it or any header is newer than its object.

    python -m ginkgo_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libginkgo_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _obj(src):
    return os.path.join(OBJ, os.path.splitext(os.path.basename(src))[0] + ".o")


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    # CUDA sources and host-only C++ sources (nvcc hands the latter to the
    # host compiler)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                  glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    jobs = []
    for s in srcs:
        o = _obj(s)
        if force or _stale(s, o, hdr_mtime):
            cmd = [nvcc, *ARCH, *FLAGS, *extra, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append((s, cmd))

    def run(job):
        s, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r

    failed = []
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for s, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                failed.append(s)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    objs = [_obj(s) for s in srcs]
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static",
               "-ldl", "-lrt", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
