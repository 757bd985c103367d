"""Builds the CUDA library and the drop-in driver in-tree.

  cosenu_b200/libcosenu_b200.so   C-ABI of include/cosenu_b200.h (sm_100a)
  cosenu_b200/bin/cosenu_main     reference-compatible driver (src/main.cpp CLI)

Objects are cached under cosenu_b200/_build/ and rebuilt when a source or
header is newer.  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libcosenu_b200.so")
BIN = os.path.join(PKG, "bin")
DRIVER = os.path.join(BIN, "cosenu_main")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
              "-ffp-contract=off", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) + \
        glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.hpp"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if _stale(obj, [src, __file__] + _headers()) or verbose_ptxas:
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj + ".tmp"]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose_ptxas:
            sys.stderr.write(r.stderr)
        os.replace(obj + ".tmp", obj)
    return obj


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC"] + objs + ["-o", LIB + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    drv_src = os.path.join(CSRC, "driver", "cosenu_main.cpp")
    if os.path.exists(drv_src) and _stale(DRIVER, [drv_src, LIB] + _headers()):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, drv_src, "-o", DRIVER + ".tmp",
               "-L", PKG, "-lcosenu_b200", "-Wl,-rpath,$ORIGIN/.."]
        subprocess.run(cmd, check=True)
        os.replace(DRIVER + ".tmp", DRIVER)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
