"""Builds the in-tree shared libraries of this package.

    python -m aretomo3_b200.build

* ``libat3r.so``        the CUDA reconstruction library (sm_100a) with the C ABI of include/at3r.h
* ``libat3r_synth.so``  the seeded phantom / tilt-series generator (host C++)
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_at3r(force: bool = False) -> str:
    out = os.path.join(PKG, "libat3r.so")
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    srcs.append(os.path.join(ROOT, "include", "at3r.h"))
    if force or _newer(out, srcs):
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include"), "-o", out, os.path.join(CSRC, "at3r.cu"),
              os.path.join(CSRC, "reproj.cu"), os.path.join(CSRC, "at3r_server.cpp"), "-ldl", "-lpthread"])
    return out


def build_synth(force: bool = False) -> str:
    out = os.path.join(PKG, "libat3r_synth.so")
    src = os.path.join(CSRC, "synth.cpp")
    if force or _newer(out, [src]):
        _run(["g++", "-O3", "-march=x86-64-v2", "-fopenmp", "-shared", "-fPIC", "-std=c++17", "-o", out, src])
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_at3r(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
