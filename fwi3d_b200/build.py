"""Build libfwi3d_b200.so in-tree with nvcc for sm_100a.

    python -m fwi3d_b200.build          (or fwi3d_b200.build.build())

CUDA sources are compiled with ``-gencode arch=compute_100a,code=sm_100a``;
host C++ sources with g++ at -O2 and no ``-march`` so their float semantics
match an x86-64 build of the reference (no FMA contraction on the host).
Objects go to fwi3d_b200/_build/, the shared library next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfwi3d_b200.so")
REPO = os.path.dirname(HERE)

CU_SOURCES = ["engine.cu", "pair.cu"]
CXX_SOURCES = ["sbp_tables.cpp", "host_ops.cpp", "capi.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cxx() -> str:
    # The plain system g++ (some images export CXX to a wrapper without OpenMP specs).
    return shutil.which("g++") or "g++"


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".inc"))]
    headers.append(os.path.join(REPO, "include", "fwi3d_gpu.h"))
    objs = []
    inc = ["-I", CSRC, "-I", os.path.join(REPO, "include")]
    jobs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                   *inc, "-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    # the CUDA translation units compile in parallel (each takes minutes)
    with ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        for f in [ex.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            _run([cxx(), "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-variable", *inc,
                  "-I", os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include"), "-c", s, "-o", o], verbose)
    if force or _stale(LIB, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lgomp"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))
