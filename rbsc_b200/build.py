"""Builds librbsc.so and the `rbsc` CLI in-tree, for sm_100a only.

    python -m rbsc_b200.build            # or: from rbsc_b200.build import build; build()

Outputs (git-ignored, but they travel with the source tree):
    rbsc_b200/librbsc.so     the C-ABI library of include/rbsc.h
    rbsc_b200/rbsc           the command-line tool with the reference's surface
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "librbsc.so")
CLI = os.path.join(PKG, "rbsc")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["rbsc.cu", "sortrelabel.cu", "gen.cu", "noalloc.cu", "batch.cu", "serve.cu", "edgebatch.cu", "lump64.cu"]
CXX_SOURCES = ["parse.cpp", "wlgen.cpp", "genhost.cpp", "bvgraph.cpp", "csrcache.cpp"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
           f"-I{os.path.join(ROOT, 'include')}"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "rbsc.h"))
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([NVCC, *ARCH, *NVFLAGS, "-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++", "-O3", "-std=c++17", "-fPIC", "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for r in ex.map(_run, jobs):
            if verbose and (r.stdout or r.stderr):
                print(r.stdout, r.stderr)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lpthread", "-ldl", "-lrt"])
    cli_src = os.path.join(CSRC, "cli.cpp")
    if force or _stale(CLI, [cli_src, LIB]):
        _run(["g++", "-O2", "-std=c++17", cli_src, "-o", CLI, f"-L{PKG}", "-lrbsc", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
