"""Build ``gbasis_b200/_lib/libgbx_eri.so`` for sm_100a (B200).

Steps: generate the class-specialised recursion sources (``csrc/gen_eri.py``) into
``csrc/_gen``, compile every ``.cu`` with nvcc in parallel, link one shared library.
Run: ``python -m gbasis_b200.build [--lmax 2] [-j 8] [--force]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "_gen")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libgbx_eri.so")
# bounds-checking build (GBX_DEBUG_BOUNDS=1): its own objects and library
BUILD_DEBUG = os.path.join(HERE, "_build_debug")
LIB_DEBUG = os.path.join(LIBDIR, "libgbx_eri_debug.so")
LMAX_DEFAULT = 3

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I", GEN] + ARCH


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources(lmax):
    sys.path.insert(0, CSRC)
    import gen_eri  # noqa: E402
    gen = gen_eri.emit_sources(GEN, lmax)
    return [os.path.join(GEN, g) for g in gen] + [
        os.path.join(CSRC, f) for f in ("runtime.cu", "pipeline.cu", "extras.cu", "noalloc.cu",
                                        "coop_kernel.cu", "batch.cu", "one_elec.cu", "boys_eval.cu")]


KERNEL_DEPS = ("gbx_common.cuh", "eri_kernels.cuh", "errors.h", "_gen/eri_gen.cuh")
HOST_DEPS = ("gbx_common.cuh", "runtime.h", "errors.h", "pipeline_kernels.cuh", "coop.cuh",
             "coop_tail.cuh", "_gen/coop_programs.cuh")


LINES_DEPS = ("gbx_common.cuh", "errors.h", "coop.cuh", "coop_tail.cuh", "lines_kernel.cuh",
              "eri_kernels.cuh", "_gen/eri_gen.cuh")


def _deps_mtime(src):
    base = os.path.basename(src)
    deps = (KERNEL_DEPS if base.startswith("eri_cls") else
            LINES_DEPS if base.startswith("lines_") else
            KERNEL_DEPS + HOST_DEPS if base in ("one_elec.cu", "boys_eval.cu") else HOST_DEPS)
    m = os.path.getmtime(os.path.join(ROOT, "include", "gbx_eri.h"))
    for d in deps:
        p = os.path.join(CSRC, d)
        if os.path.exists(p):
            m = max(m, os.path.getmtime(p))
    return m


def compile_one(src, force, verbose_ptxas=False, debug=False):
    obj = os.path.join(BUILD_DEBUG if debug else BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(
            os.path.getmtime(src), _deps_mtime(src)):
        return obj, 0.0, ""
    cmd = [nvcc(), *NVCC_FLAGS, *(["-DGBX_DEBUG_BOUNDS=1"] if debug else []), "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    t = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-6000:]}")
    return obj, time.time() - t, r.stderr


def build(lmax=LMAX_DEFAULT, jobs=None, force=False, verbose=False, ptxas=False, debug=False):
    """Build the library; ``debug``: the bounds-checking one (libgbx_eri_debug.so)."""
    lib_path = LIB_DEBUG if debug else LIB
    os.makedirs(BUILD_DEBUG if debug else BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources(lmax)
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    objs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, dt, err in ex.map(lambda s: compile_one(s, force, ptxas, debug), srcs):
            objs.append(obj)
            if verbose and dt:
                print(f"  {os.path.basename(obj)}: {dt:.1f}s", flush=True)
            if ptxas and err:
                print(err)
    if force or not os.path.exists(lib_path) or os.path.getmtime(lib_path) < max(
            os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib_path, *objs, "-lcublas", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return lib_path


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--lmax", type=int, default=LMAX_DEFAULT)
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    ap.add_argument("--debug-bounds", action="store_true",
                    help="build libgbx_eri_debug.so with every kernel store index-checked")
    a = ap.parse_args()
    t = time.time()
    print(build(a.lmax, a.j, a.force, verbose=True, ptxas=a.ptxas, debug=a.debug_bounds),
          f"{time.time() - t:.1f}s")
