"""Builds the in-tree CUDA library ``eos_b200/libeos_b200.so`` for sm_100a with nvcc.

Every translation unit is compiled with ``--fmad=false``: the render path reproduces the
reference CPU renderer's float rounding operation by operation, so a*b + c must stay a
rounded multiply followed by a rounded add (kernels that want an FMA ask for one
explicitly).  Division and sqrt keep their IEEE defaults (no fast-math).

    python -m eos_b200.build [--force] [--verbose-ptxas]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libeos_b200.so")
SOURCES = ["api.cu", "lbvh.cu", "ploc.cu", "instances.cu", "scene_io.cu", "render.cu", "wavefront.cu", "adjoint.cu", "mesh.cpp"]
HEADERS = ["eos_math.cuh", "eos_internal.cuh", "trace.cuh", "scan.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _flags(verbose_ptxas: bool) -> list[str]:
    f = ARCH + ["-lineinfo", "-O3", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
                "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "eos_c.h")]
    newest_dep = max(_mtime(d) for d in deps)
    objs, jobs = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OUT_DIR, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if force or verbose_ptxas or _mtime(obj) < max(_mtime(src), newest_dep):
            jobs.append([nvcc(), "-c", src, "-o", obj] + _flags(verbose_ptxas))
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
    for c, r in zip(jobs, results):
        if verbose_ptxas or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(c)}")
    if force or jobs or not os.path.exists(LIB) or _mtime(LIB) < max(_mtime(o) for o in objs):
        tmp = LIB + ".tmp"
        # -z defs: a symbol left undefined fails the link instead of the first load
        cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC", "-cudart", "static",
                                                             "-Xlinker", "-z", "-Xlinker", "defs"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose_ptxas))
