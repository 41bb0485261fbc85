"""Build libcellsb200.so in-tree with nvcc for sm_100a (the only target).

    python -m cells_b200.build [--force]
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = [os.path.join(HERE, "csrc", "tissue_step.cu")]
HEADERS = [os.path.join(ROOT, "include", "cells_b200.h")]
OUTPUT = os.path.join(HERE, "libcellsb200.so")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-shared", "-Xcompiler", "-fPIC",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date():
    if not os.path.exists(OUTPUT):
        return False
    built = os.path.getmtime(OUTPUT)
    return all(os.path.getmtime(p) <= built for p in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUTPUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUTPUT, *SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUTPUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=True))
    return 0


if __name__ == "__main__":
    sys.exit(main())
