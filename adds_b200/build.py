"""Builds libadds.so (sm_100a) and the drop-in CLIs in-tree.

Outputs (git-ignored, shipped with the tree):
  adds_b200/lib/libadds.so         the C ABI of include/adds.h
  adds_b200/bin/sssp_int           drop-in for the reference ads_int/sssp
  adds_b200/bin/sssp_float         drop-in for the reference ads_float/sssp

Every CUDA translation unit is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with -fmad=false so that no
multiply-add contraction can change a float sum.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
BINDIR = os.path.join(HERE, "bin")
LIB = os.path.join(LIBDIR, "libadds.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include")]
CU_SOURCES = ["engine.cu", "phase.cu", "api.cu", "gen.cu", "adjoint.cu", "noalloc.cu", "diag.cu"]
CXX_SOURCES = ["grio.cpp"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_nvcc=None) -> str:
    """Compiles what changed; returns the path of libadds.so."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    headers = [os.path.join(CSRC, "adds_internal.h"), os.path.join(CSRC, "phase_internal.h"),
               os.path.join(ROOT, "include", "adds.h")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([NVCC] + NVCC_FLAGS + (extra_nvcc or []) + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-pthread",
                         "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart", "-lpthread"], verbose)
        os.replace(tmp, LIB)
    cli = os.path.join(CSRC, "sssp_cli.c")
    for name, defs in (("sssp_int", []), ("sssp_float", ["-DADDS_CLI_FLOAT"])):
        exe = os.path.join(BINDIR, name)
        if force or _stale(exe, [cli, LIB, headers[-1]]):
            _run(["gcc", "-O2", "-std=c11", "-Wall", "-D_POSIX_C_SOURCE=200809L"] + defs +
                 ["-I", os.path.join(ROOT, "include"), cli, "-o", exe, "-L", LIBDIR, "-ladds",
                  "-Wl,-rpath,$ORIGIN/../lib"], verbose)
    return LIB


def clean():
    for d in (BUILD, LIBDIR, BINDIR):
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
