"""Build ``libdglm.so`` in-tree with nvcc for sm_100a.

Usage: ``python -m exadglm_b200.build [--force] [-j N]``.  Objects go to
``_build/``; the library lands next to this file so it travels with the
working tree.  Compilation is incremental on source/header mtimes.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libdglm.so")
MAIN_SRC = os.path.join(CSRC, "host", "dglm_main.cpp")
MAIN = os.path.join(PKG, "dglm_main")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
              "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _compile(src, force):
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and \
            os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps()):
        return obj, None
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}")
    return obj, r.stdout


def build(force=False, jobs=None, verbose=False):
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, out in results:
            if out:
                print(out)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        # static cudart: the library carries its own 12.9 runtime and shares
        # the device's primary context with any other runtime in the process
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
        os.replace(tmp, LIB)
    if force or not os.path.exists(MAIN) or \
            os.path.getmtime(MAIN) < max(os.path.getmtime(LIB), os.path.getmtime(MAIN_SRC)):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, MAIN_SRC, "-o", MAIN + ".tmp",
               "-L", PKG, "-ldglm", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("dglm_main build failed:\n" + r.stdout)
        os.replace(MAIN + ".tmp", MAIN)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.j, verbose=a.v))
    return 0


if __name__ == "__main__":
    sys.exit(main())
