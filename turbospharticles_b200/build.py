"""Builds the in-tree CUDA library `_build/libtsp_b200.so` for sm_100a with nvcc.

    python -m turbospharticles_b200.build [--force]

-fmad=false: every multiply-add in the kernels is written out (fmaf where the reference
uses fma), so per-pair arithmetic follows the reference's operation order exactly.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

from .abi import LIB_PATH, PKG_DIR

CSRC = os.path.join(PKG_DIR, "csrc")
SOURCES = ["backend.cu", "ns_kernels.cu", "sph_kernels.cu", "rigid_kernels.cu", "noalloc.cu", "batch.cu", "contact_kernels.cu", "stats_kernels.cu", "export_kernels.cu", "surface_kernels.cu", "tune.cu"]
HEADERS = ["common.cuh", "kernels.h", "primitives.cuh", "host_common.h"]
INCLUDE = os.path.join(os.path.dirname(PKG_DIR), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> str:
    build_dir = os.path.dirname(LIB_PATH)
    os.makedirs(build_dir, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "tsp_b200.h")]
    objs = []
    host_cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else None
    cmds = []
    for src in SOURCES:
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, deps):
            cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *extra_flags, "-I", INCLUDE, "-c",
                   os.path.join(CSRC, src), "-o", obj]
            if host_cxx:
                cmd[1:1] = ["-ccbin", host_cxx]
            if verbose:
                print(" ".join(cmd))
            cmds.append(cmd)
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or _stale(LIB_PATH, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB_PATH, *objs, "-lcudart"]
        if host_cxx:
            cmd[1:1] = ["-ccbin", host_cxx]
        subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB_PATH)
