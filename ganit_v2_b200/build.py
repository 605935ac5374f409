"""Build recipe of libganit_b200.so (sm_100a only).

``python -m ganit_v2_b200.build`` compiles every CUDA source in csrc/ with
nvcc into ganit_v2_b200/libganit_b200.so, in the source tree, so the library
travels with the repository.  No torch extension machinery is involved: the
library exposes a plain C ABI (include/ganit_b200.h).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libganit_b200.so")
SOURCES = ["gb_engine.cu", "gb_backend.cu", "gb_diff.cu", "gb_noalloc.cu", "gb_pool.cu", "gb_branch.cu", "gb_mps.cpp", "gb_factor.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "ganit_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, jobs: int = 4) -> str:
    """Compile (when sources are newer than the library) and return its path."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    cc = nvcc()
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmd = [cc, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        if len(procs) >= jobs:
            _wait(procs.pop(0), verbose)
    for p in procs:
        _wait(p, verbose)
    link = [cc, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    out = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if out.returncode != 0:
        raise RuntimeError("link failed:\n" + out.stdout)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def _wait(item, verbose):
    src, p = item
    out, _ = p.communicate()
    if verbose and out:
        print(out)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{out}")


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
