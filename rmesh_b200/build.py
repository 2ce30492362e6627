"""Builds ``rmesh_b200/lib/librmesh_b200.so`` from ``rmesh_b200/csrc`` with nvcc.

Usage: ``python -m rmesh_b200.build`` (cross-compiles for sm_100a; no GPU needed).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "librmesh_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # IEEE division and square root (the exact per-tet stages also use explicit __f*_rn)
    "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-shared",
]


def nvcc_path() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources_newer_than(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    for root in (SRC, os.path.join(os.path.dirname(HERE), "include")):
        for f in os.listdir(root):
            if os.path.getmtime(os.path.join(root, f)) > t:
                return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not sources_newer_than(OUT):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc_path(), *NVCC_FLAGS, "-o", OUT, os.path.join(SRC, "api.cu")]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building librmesh_b200.so")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
