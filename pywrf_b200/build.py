"""Build the sm_100a kernel library in-tree.

``python -m pywrf_b200.build`` compiles every ``csrc/*.cu`` with nvcc for
``sm_100a`` (``-gencode arch=compute_100a,code=sm_100a``) and links
``pywrf_b200/lib/libpywrf_b200.so``.  No JIT cache is involved: the built
library lives next to the sources and is what :mod:`pywrf_b200._native`
loads.  Objects go to ``pywrf_b200/_build``; a source is recompiled when it or
any header is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libpywrf_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the reference rounds every multiply and add separately; letting
# nvcc contract them into FMAs changes the rounding of the many
# cancellation-prone differences of the step (bdy - ph*mu, muts*t_1 - mut*t_2,
# p0*pp - pb ...) for no measurable gain in these memory-bound kernels.
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                     "-I" + INCLUDE, "-I" + CSRC]
# the network's tensor-core products have no reference operation order to
# follow: their epilogues may contract multiply-adds
FMAD_SOURCES = {"k_gemm_tc.cu"}


def flags_for(src: str) -> list[str]:
    if os.path.basename(src) in FMAD_SOURCES:
        return [f if f != "-fmad=false" else "-fmad=true" for f in NVCC_FLAGS]
    return list(NVCC_FLAGS)


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the sm_100a kernels cannot be built")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(src: str, obj: str, hdr_mtime: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or hdr_mtime > t


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    """Compile and link the library; returns its path."""
    nvcc = nvcc_path()
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    if not srcs:
        raise RuntimeError("no CUDA sources under " + CSRC)
    hdr_mtime = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(s, o, hdr_mtime)]

    def compile_one(so):
        s, o = so
        cmd = [nvcc] + flags_for(s) + (["-Xptxas", "-v"] if verbose else []) + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n{r.stderr}")
        return s, r.stderr

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for s, log in ex.map(compile_one, todo):
                if verbose and log:
                    sys.stderr.write(f"== {os.path.basename(s)}\n{log}")
    if force or todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr)
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill reports")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
