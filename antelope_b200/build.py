"""Build recipe of the native library (run by __graft_entry__.build()).

Compiles the sm_100a kernels and the C++ host code into
antelope_b200/libsbe_b200.so (the C ABI of include/sbe.h) and the
command-line drop-in antelope_b200/bin/sbe_run.  nvcc cross-compiles for
sm_100a without a GPU.  Objects go to antelope_b200/_build/.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsbe_b200.so")
CLI = os.path.join(HERE, "bin", "sbe_run")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O2,-Wall"]
SOURCES = ["sbe_kernels.cu", "sbe_problem.cpp", "sbe_engine.cpp", "sbe_capi.cpp", "sbe_noalloc.cu", "sbe_tune.cpp", "sbe_wannier.cu", "sbe_wansolve.cpp", "sbe_materials.cpp", "sbe_spectrum.cu"]
HEADERS = ["sbe_dev.h", "sbe_kernels.h", "sbe_problem.h", "sbe_engine.h", "sbe_handles.h", "sbe_wannier.h", "sbe_wansolve.h", "sbe_spectrum.h", "sbe_wangroup.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "sbe.h")]
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer(o, [s, __file__] + hdrs):
            extra = ["-Xptxas", "-v"] if (verbose_ptxas and src.endswith(".cu")) else []
            jobs.append([NVCC] + ARCH + COMMON + extra + ["-c", s, "-o", o])
    # the translation units are independent: compile them in parallel
    if jobs:
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as pool:
            for f in [pool.submit(_run, cmd) for cmd in jobs]:
                f.result()
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    cli_src = os.path.join(CSRC, "sbe_run.cpp")
    if _newer(CLI, [cli_src, LIB]):
        _run(["g++", "-O2", "-std=c++17", "-o", CLI, cli_src, "-L" + HERE, "-lsbe_b200",
              "-Wl,-rpath,$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
