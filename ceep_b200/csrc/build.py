"""Build ``ceep_b200/_lib/libceep_b200.so`` from the CUDA sources in this folder.

    python -m ceep_b200.csrc.build            # or: python ceep_b200/csrc/build.py
    python -m ceep_b200.csrc.build --incremental   # only the sources that changed

Compiles for sm_100a only (B200), statically linking the CUDA runtime so the
library does not depend on a particular libcudart on the loader path.  With
``--ptxas-info`` the ptxas register/spill report of every kernel is printed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libceep_b200.so")
# the 2D forward kernels compile once per ADE shape (fdtd2d_d<ND>l<NL>.cu)
FDTD2D_SHAPES = ["fdtd2d_d0l0.cu", "fdtd2d_d0l1.cu", "fdtd2d_d0l2.cu", "fdtd2d_d1l0.cu", "fdtd2d_d1l1.cu",
                 "fdtd2d_d2l0.cu"]
SOURCES = ["capi.cu", "fdtd2d.cu"] + FDTD2D_SHAPES + ["fdtd3d.cu", "adjoint2d.cu", "adjoint3d.cu", "spectral.cu",
                                                      "phantom.cu", "single2d.cu", "materials.cu"]
HEADERS = ["common.cuh", "fdtd2d.cuh", "fdtd2d_kernels.cuh", "fdtd3d.cuh", "adjoint2d.cuh", "adjoint3d.cuh",
           "tma.cuh", "capi_internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "ceep_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


OBJ_DIR = os.path.join(OUT_DIR, "obj")


def _obj_stale(src: str, obj: str) -> bool:
    """An object is rebuilt when it is missing or older than its source or
    than any shared header."""
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [os.path.join(HERE, src)] + [os.path.join(HERE, h) for h in HEADERS] + \
        [os.path.join(ROOT, "include", "ceep_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, ptxas_info: bool = False, verbose: bool = False) -> str:
    """Compile the sources that changed (every one with `force` or
    `ptxas_info`), in parallel, and link the library.  Objects are kept in
    _lib/obj so that a change to one source recompiles only that one."""
    if not force and not ptxas_info and not _stale():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    # -compress-all: the per-shape fatbins with line info are otherwise stored uncompressed (~3x larger)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                    "-Xfatbin", "-compress-all"]
    if ptxas_info:
        flags += ["-Xptxas", "-v"]
    objs = [os.path.join(OBJ_DIR, src.replace(".cu", ".o")) for src in SOURCES]
    todo = [(src, obj) for src, obj in zip(SOURCES, objs) if force or ptxas_info or _obj_stale(src, obj)]

    def compile_one(job):
        src, obj = job
        cmd = [nvcc()] + flags + ["-c", os.path.join(HERE, src), "-o", obj + ".tmp"]
        if verbose:
            print(" ".join(cmd))
        return src, obj, subprocess.run(cmd, capture_output=True, text=True)

    # one nvcc per source, in parallel (the translation units are independent)
    workers = max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as pool:
        results = list(pool.map(compile_one, todo))
    for src, obj, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if ptxas_info:
            sys.stdout.write(r.stderr)
        os.replace(obj + ".tmp", obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    print(build(force="--incremental" not in args, ptxas_info="--ptxas-info" in args, verbose="-v" in args))
