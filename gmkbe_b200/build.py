"""Build the in-tree native artefacts.

    python -m gmkbe_b200.build          # libgmk.so + the gmk CLI (sm_100a), gmk-convert

Everything is compiled with nvcc for sm_100a only and written next to the
sources (gmkbe_b200/libgmk.so, gmkbe_b200/gmk), so the built files travel with
a copy of the repository.
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
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-I" + os.path.join(ROOT, "include")]

LIB = os.path.join(PKG, "libgmk.so")
CLI = os.path.join(PKG, "gmk")
CONVERT = os.path.join(PKG, "gmk-convert")
CXX = os.environ.get("CXX", "g++")


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False) -> None:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "gmk.h")]
    if force or _stale(LIB, deps):
        _run([NVCC, *ARCH, *COMMON, "-Xcompiler", "-fPIC", "-shared", "-o", LIB,
              os.path.join(CSRC, "gmk_capi.cu")])
    if force or _stale(CLI, deps + [LIB]):
        _run([NVCC, *ARCH, *COMMON, "-o", CLI, os.path.join(CSRC, "gmk_cli.cpp"),
              "-L" + PKG, "-lgmk", "-Xlinker", "-rpath=$ORIGIN"])
    conv_src = os.path.join(CSRC, "gmk_convert.cpp")
    if force or _stale(CONVERT, [conv_src]):
        _run([CXX, "-O3", "-std=c++17", "-pthread", "-o", CONVERT, conv_src])


if __name__ == "__main__":
    build(force="--force" in sys.argv)
