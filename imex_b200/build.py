"""Build recipe of libimex_b200.so (sm_100a) and the two oracle libraries.

``build_library()`` compiles every CUDA source of imex_b200/csrc with nvcc for
sm_100a into ``imex_b200/libimex_b200.so`` (in-tree, so it travels with the
repository snapshot).  FMA contraction is disabled (``-fmad=false``) so that
the FP64 kernels round exactly like the reference's x86 build.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libimex_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers() -> list[str]:
    return (sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")))
            + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh")))
            + [os.path.join(ROOT, "include", "imex_b200.h")])


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    srcs = sources()
    if not force and not _stale(LIB, srcs + headers()):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(out)
        elif verbose and out.strip():
            sys.stderr.write(out)
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


DRIVER_SRC = os.path.join(HERE, "driver", "imex_run.cpp")
DRIVER = os.path.join(HERE, "imex_run")


def build_driver(force: bool = False) -> str:
    """The time-marching driver executable (C++ over the C ABI), linked to the in-tree library."""
    if not force and not _stale(DRIVER, [DRIVER_SRC, LIB, os.path.join(ROOT, "include", "imex_b200.h")]):
        return DRIVER
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), DRIVER_SRC,
           "-L", HERE, "-limex_b200", "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    subprocess.run(cmd, check=True)
    return DRIVER


def build_oracles() -> None:
    """Build oracle/liboracle.so always, oracle/_ref when the reference sources exist
    (oracle/Makefile knows where they lie; `make have-ref` says whether they are there)."""
    oracle = os.path.join(ROOT, "oracle")
    subprocess.run(["make", "-s", "-C", oracle, "port"], check=True)
    if subprocess.run(["make", "-s", "-C", oracle, "have-ref"], stdout=subprocess.DEVNULL,
                      stderr=subprocess.DEVNULL).returncode == 0:
        subprocess.run(["make", "-s", "-C", oracle, "ref"], check=True)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_driver(force="--force" in sys.argv)
    build_oracles()
