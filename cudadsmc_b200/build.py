"""Build recipes for the in-tree native libraries.

* ``libdsmc_b200.so`` -- the sm_100a engine and its C ABI (``include/dsmc.h``), built with
  nvcc ``-gencode arch=compute_100a,code=sm_100a``.  Device code is compiled with
  ``--fmad=false`` so that no multiply-add is contracted behind the program's back: every
  operation of the timestep is the correctly rounded IEEE operation written in the source,
  which is what lets the CPU oracle reproduce the GPU bit for bit.
* ``oracle/build/liboracle.so`` -- the CPU restatement used by the tests and the CPU
  baseline (g++, OpenMP, ``-ffp-contract=off``).

Both land inside the repository tree so that they travel with it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(ROOT, "include")
ENGINE_SO = os.path.join(PKG_DIR, "libdsmc_b200.so")
DRIVER_BIN = os.path.join(PKG_DIR, "dsmc_driver")
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "build", "liboracle.so")

ENGINE_SOURCES = ["dsmc_engine.cu", "dsmc_noalloc.cu"]
ENGINE_HEADERS = ["dsmc_kernels.cuh", "dsmc_physics.h", "dsmc_radix.cuh", "dsmc_setup.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]

# x86-64-v3 (AVX2 + FMA): the oracle library is built here and run on the GPU host
ORACLE_CXXFLAGS = [
    "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-math-errno", "-fopenmp",
    "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the system g++ ships libgomp; wrapper compilers earlier on PATH may not
    for cand in ("/usr/bin/g++", os.environ.get("CXX"), shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")


def build_engine(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in ENGINE_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in ENGINE_HEADERS] + [os.path.join(INCLUDE, "dsmc.h")]
    if force or _stale(ENGINE_SO, deps):
        cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-shared", "-o", ENGINE_SO, *srcs]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        _run(cmd)
    return ENGINE_SO


def build_driver(force: bool = False) -> str:
    """The command-line driver (csrc/driver.cpp) linked against libdsmc_b200.so."""
    src = os.path.join(CSRC, "driver.cpp")
    if force or _stale(DRIVER_BIN, [src, ENGINE_SO, os.path.join(INCLUDE, "dsmc.h")]):
        _run([_cxx(), "-O2", "-std=c++17", "-I", INCLUDE, "-o", DRIVER_BIN, src, "-L", PKG_DIR, "-ldsmc_b200",
              "-Wl,-rpath,$ORIGIN"])
    return DRIVER_BIN


def build_oracle(force: bool = False) -> str:
    src = os.path.join(ORACLE_DIR, "dsmc_oracle.cpp")
    deps = [src] + [os.path.join(CSRC, h) for h in ("dsmc_physics.h", "dsmc_setup.h")] + [os.path.join(INCLUDE, "dsmc.h")]
    if force or _stale(ORACLE_SO, deps):
        os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
        cxx = _cxx()
        _run([cxx, *ORACLE_CXXFLAGS, "-I", INCLUDE, "-I", CSRC, "-o", ORACLE_SO, src])
    return ORACLE_SO


def build_all(force: bool = False) -> None:
    build_engine(force)
    build_driver(force)
    build_oracle(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ENGINE_SO)
    print(ORACLE_SO)
