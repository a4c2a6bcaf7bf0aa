"""In-tree build of the native libraries.

    python -m gems_b200.build          # builds what is out of date

libgems_b200.so  -- CUDA kernels (sm_100a) + C-ABI session layer + host tree mirror
libgems_synth.so -- host C synthetic-workload generator

Both land next to this file so they travel with the repository snapshot.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]

CUDA_SOURCES = ["session.cu", "kernels_fp64.cu", "kernels_mixed.cu", "kernels_traverse.cu",
                "kernels_tc20.cu", "kernels_tc61.cu", "kernels_g61.cu", "kernels_rell.cu", "eigen.cu", "noalloc.cu", "peaks.cu", "ingest.cu",
                "phylotree.cpp"]
HEADERS = ["gems_internal.cuh", "tc_common.cuh", "plan.h"]

LIB = os.path.join(HERE, "libgems_b200.so")
SYNTH = os.path.join(HERE, "libgems_synth.so")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build failed: " + os.path.basename(cmd[-1]))
    return r


def build_synth(force=False):
    src = os.path.join(CSRC, "synth.c")
    if force or _newer(SYNTH, [src]):
        _run(["gcc", "-O2", "-fPIC", "-fopenmp", "-shared", "-o", SYNTH, src, "-lm"])
    return SYNTH


def build_cuda(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "gems_b200.h")]
    objs, jobs = [], []
    for src in CUDA_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path] + hdrs):
            jobs.append([NVCC] + NVFLAGS + (["-Xptxas", "-v"] if verbose else []) +
                        ["-c", path, "-o", obj])
    # translation units compile independently: one nvcc per source, in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in ex.map(_run, jobs):
            if verbose:
                sys.stderr.write(r.stderr)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


def build_all(force=False, verbose=False):
    build_synth(force)
    build_cuda(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
    print(SYNTH)
