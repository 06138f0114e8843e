"""Build recipe of the CUDA extension: nvcc for sm_100a, in-tree output.

``python -m nrqcd_b200.build`` compiles every translation unit under
``nrqcd_b200/csrc`` with ``-gencode arch=compute_100a,code=sm_100a`` and
links ``nrqcd_b200/_lib/libnrqcd_b200.so`` (plain C ABI of
``include/nrqcd_b200.h``).  nvcc cross-compiles without a GPU.
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
OUT_DIR = os.path.join(HERE, "_lib")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libnrqcd_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra_flags=None, ptxas_verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "nrqcd_b200.h"))
    flags = FLAGS + list(extra_flags or [])
    if ptxas_verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    jobs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if ptxas_verbose or _newer(obj, [src] + headers):
            jobs.append([nvcc(), *ARCH, *flags, "-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or ptxas_verbose:
                sys.stdout.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    # objects of translation units that no longer exist force a relink
    stale = [f for f in os.listdir(BUILD_DIR) if f.endswith(".o") and os.path.join(BUILD_DIR, f) not in objs]
    for f in stale:
        os.remove(os.path.join(BUILD_DIR, f))
    if stale or _newer(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv))
