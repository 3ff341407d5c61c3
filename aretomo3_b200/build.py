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
    """Compiles the CUDA / C++ sources to objects in parallel (csrc/_build/),
    then links libat3r.so."""
    out = os.path.join(PKG, "libat3r.so")
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    srcs.append(os.path.join(ROOT, "include", "at3r.h"))
    if not (force or _newer(out, srcs)):
        return out
    units = ["at3r.cu", "reproj.cu", "stack.cu", "at3r_server.cpp", "mrc.cpp"]
    bdir = os.path.join(CSRC, "_build")
    os.makedirs(bdir, exist_ok=True)
    common = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
    procs, objs = [], []
    for u in units:
        obj = os.path.join(bdir, u.rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        cmd = [*common, "-c", os.path.join(CSRC, u), "-o", obj]
        print(" ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd))
    if any(p.wait() != 0 for p in procs):
        raise subprocess.CalledProcessError(1, "nvcc")
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-ldl", "-lpthread"])
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
