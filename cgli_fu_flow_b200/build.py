"""Builds the CUDA library libcgli_fu_flow.so in-tree for sm_100a.

The library is the product: every kernel of the hot path and the C ABI of
include/cgli_fu_flow.h.  Compiled with nvcc for sm_100a only; it is built
in the package directory so it travels with the repository snapshot.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcgli_fu_flow.so")
DRIVER = os.path.join(HERE, "cgli_run")                 # the C++ host driver (csrc/driver)
DRIVER_SRC = os.path.join(HERE, "csrc", "driver", "cgli_run.cpp")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xptxas", "-warn-spills"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cpp")))


def deps() -> list[str]:
    return sources() + glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        [os.path.join(REPO, "include", "cgli_fu_flow.h"), os.path.abspath(__file__)]


def build_driver(force: bool = False) -> str:
    """The C++ host driver (main.cpp's step loop on the C ABI), linked
    against the in-tree library with an $ORIGIN run path."""
    if not force and os.path.exists(DRIVER) and all(
            os.path.getmtime(d) <= os.path.getmtime(DRIVER) for d in (DRIVER_SRC, LIB)):
        return DRIVER
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(REPO, "include"), DRIVER_SRC,
                    "-L", HERE, "-lcgli_fu_flow", "-Wl,-rpath,$ORIGIN", "-o", DRIVER], check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps()):
        build_driver()
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(REPO, "include"), "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            sys.stderr.write(out.decode())
        if p.returncode:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], check=True)
    build_driver(force=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
