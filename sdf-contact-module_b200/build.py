"""Builds libsdfo_cuda.so (sm_100a) in-tree from csrc/*.cu.

    python sdf-contact-module_b200/build.py [--force] [--verbose]

Each translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; build.cu and
batch.cu, ca_build.cu, ca_query.cu and be_step.cu (the FP64 distance / sign /
candidate / integrator paths) additionally with ``-fmad=false`` so their FP64
expressions are evaluated exactly in source order.  The static CUDA runtime
is linked in so the library does not depend on the toolkit's libcudart at
run time.  Objects go to _build/, the library to lib/.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libsdfo_cuda.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
          "-ffp-contract=off", "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
PER_FILE = {"build.cu": ["-fmad=false"], "batch.cu": ["-fmad=false"], "ca_build.cu": ["-fmad=false"],
            "ca_query.cu": ["-fmad=false"], "be_step.cu": ["-fmad=false"]}
SOURCES = ["grid.cu", "capi.cu", "query.cu", "build.cu", "batch.cu", "batch_query.cu",
           "ca_build.cu", "ca_query.cu", "contact.cu", "static_staging.cu", "sdfo_file.cu",
           "contact_pair.cu", "be_step.cu", "stream_bwd.cu", "host_query.cu"]
HEADERS = ["sdfo_internal.cuh", "interp.cuh", "build_common.cuh", "bulk.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "sdfo.h"),
                                                    os.path.abspath(__file__)]
    # extra nvcc flags from the environment (e.g. -DSDFO_QUERY_SPARSE_MIN_BLOCKS=4
    # to try another register budget); they are part of the objects' inputs,
    # so a change forces a rebuild
    env_flags = os.environ.get("SDFO_NVCC_FLAGS", "").split()
    stamp = os.path.join(BUILD, "flags.txt")
    flags_now = " ".join(env_flags + (extra_flags or []))
    if not os.path.exists(stamp) or open(stamp).read() != flags_now:
        force = True
        with open(stamp, "w") as f:
            f.write(flags_now)
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdr):
            cmd = [nvcc(), "-c", s, "-o", o] + ARCH + COMMON + PER_FILE.get(src, []) + env_flags + (extra_flags or [])
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-cudart", "static",
                                                            "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_host(force, verbose)
    return LIB


HOST = os.path.join(PKG, "host")
HOST_LIB = os.path.join(LIBDIR, "libsdfo_host.so")
HOST_CHECK = os.path.join(LIBDIR, "sdfo_host_check")
HOST_SOURCES = ["SdfIO.cpp", "SdfSurfaceMesh.cpp", "SdfBuilder.cpp", "SdfOracle.cpp"]


def host_cxx() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def build_host(force: bool = False, verbose: bool = False) -> str:
    """The C++ plugin API (libsdfo_host.so) and its check program, linked
    against libsdfo_cuda.so with an $ORIGIN run path."""
    hdrs = [os.path.join(HOST, "include", "SdfOracle", h)
            for h in os.listdir(os.path.join(HOST, "include", "SdfOracle"))]
    hdrs += [os.path.join(INCLUDE, "sdfo.h"), os.path.join(HOST, "compat", "Eigen", "Dense")]
    flags = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-I", os.path.join(HOST, "include"),
             "-I", os.path.join(HOST, "compat"), "-I", INCLUDE]
    srcs = [os.path.join(HOST, "src", s) for s in HOST_SOURCES]
    link = ["-L", LIBDIR, "-lsdfo_cuda", "-Wl,-rpath,$ORIGIN"]
    if force or _newer(HOST_LIB, srcs + hdrs + [LIB]):
        cmd = [host_cxx(), "-shared", "-o", HOST_LIB] + flags + srcs + link
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    app = os.path.join(HOST, "app", "sdfo_host_check.cpp")
    if force or _newer(HOST_CHECK, [app, HOST_LIB] + hdrs):
        cmd = [host_cxx(), "-o", HOST_CHECK, app] + flags + ["-L", LIBDIR, "-lsdfo_host"] + link
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return HOST_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else None
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose, extra_flags=extra))
    sys.exit(0)
