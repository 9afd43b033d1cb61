"""Build libgrid_b200.so (sm_100a CUDA layer + C host layer) in-tree.

Usage: python -m libgrid_b200.build [--force] [-j N]

Objects go to libgrid_b200/_build/, the shared library to
libgrid_b200/libgrid_b200.so.  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgrid_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE] + ARCH
CC_FLAGS = ["-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wno-unused-function", "-I" + INCLUDE]


def _sources():
    cu = sorted(
        os.path.join(CSRC, "cuda", f) for f in os.listdir(os.path.join(CSRC, "cuda")) if f.endswith(".cu")
    )
    c = sorted(os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host")) if f.endswith(".c"))
    return cu, c


def _headers():
    hs = []
    for d in (os.path.join(CSRC, "cuda"), os.path.join(CSRC, "host"), INCLUDE):
        hs += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return hs


def _obj(src):
    return os.path.join(BUILD, os.path.basename(src) + ".o")


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
    return p.stdout + p.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cu, c = _sources()
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    cmds = []
    for s in cu:
        o = _obj(s)
        if force or _stale(s, o, hdr_mtime):
            cmds.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    for s in c:
        o = _obj(s)
        if force or _stale(s, o, hdr_mtime):
            cmds.append(["gcc"] + CC_FLAGS + ["-c", s, "-o", o])
    jobs = jobs or min(8, os.cpu_count() or 4)
    if cmds:
        with cf.ThreadPoolExecutor(jobs) as ex:
            for out in ex.map(_run, cmds):
                if verbose and out.strip():
                    print(out)
    objs = [_obj(s) for s in cu + c]
    if force or cmds or not os.path.exists(LIB):
        _run([NVCC, "-shared", "-cudart", "static"] + ARCH + ["-o", LIB] + objs + ["-lm"])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    sys.exit(main())
