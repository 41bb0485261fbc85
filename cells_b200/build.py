"""Build libcellsb200.so in-tree with nvcc for sm_100a (the only target).

    python -m cells_b200.build [--force]

Each translation unit of csrc/ compiles to an object under csrc/_build/ (in parallel); the
objects link into cells_b200/libcellsb200.so. A unit recompiles when it, a csrc header or the
public header is newer than its object.
"""

from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SOURCES = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
OBJDIR = os.path.join(CSRC, "_build")
OUTPUT = os.path.join(HERE, "libcellsb200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                  + [os.path.join(ROOT, "include", "cells_b200.h")])


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _object(src):
    return os.path.join(OBJDIR, os.path.splitext(os.path.basename(src))[0] + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    built = os.path.getmtime(target)
    return any(os.path.getmtime(p) > built for p in deps)


def up_to_date():
    objs = [_object(s) for s in SOURCES]
    return not any(_stale(o, [s, *headers()]) for s, o in zip(SOURCES, objs)) and not _stale(
        OUTPUT, objs)


def build(force=False, verbose=False):
    os.makedirs(OBJDIR, exist_ok=True)
    deps = headers()
    jobs = []
    for src in SOURCES:
        obj = _object(src)
        if force or _stale(obj, [src, *deps]):
            jobs.append([nvcc(), *COMPILE_FLAGS, "-c", "-o", obj, src])
    if verbose:
        for cmd in jobs:
            print(" ".join(cmd))
    with ThreadPoolExecutor(max(1, len(jobs))) as pool:
        results = list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
    for cmd, res in zip(jobs, results):
        if res.stdout or res.stderr:
            sys.stderr.write(res.stdout + res.stderr)
        if res.returncode:
            raise subprocess.CalledProcessError(res.returncode, cmd)
    objs = [_object(s) for s in SOURCES]
    if force or jobs or _stale(OUTPUT, objs):
        link = [nvcc(), *ARCH, "-shared", "-o", OUTPUT, *objs]
        if verbose:
            print(" ".join(link))
        subprocess.run(link, check=True)
    return OUTPUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=True))
    return 0


if __name__ == "__main__":
    sys.exit(main())
