"""Build libnbc.so (the engine and its C ABI) in-tree for sm_100a.

    python nbody-clump_b200/build.py [--force] [--verbose]

nvcc compiles the CUDA sources and the C++ host files with
`-gencode arch=compute_100a,code=sm_100a`; the shared library lands next to
this file so it travels with the source tree.  No GPU is needed to build.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libnbc.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "capi.cpp", "io.cpp", "noalloc.cu", "tune.cpp", "serve.cpp", "generate.cu"]
HEADERS = ["kernels.cuh", "nbc_dev.cuh", "nbc_math.cuh", "engine.h", "io.h", "handle.h", "dem_clump_main.h",
           "dem_clump_main.cpp", "main.cpp", "dem_main.h", "dem_main.cpp", "sphere_main.cpp"]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "nbc.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    objs = []
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "-I", os.path.join(os.path.dirname(HERE), "include")]
    # extra nvcc flags, e.g. NBC_NVCC_FLAGS="-DNBC_PAIR_MINB=3" for another
    # launch-bounds choice of the pair kernel
    common += os.environ.get("NBC_NVCC_FLAGS", "").split()
    for src in SOURCES:
        obj = os.path.join(CSRC, "_obj_" + src.replace(".", "_") + ".o")
        lang = [] if src.endswith(".cu") else ["-x", "cu"] if src.endswith(".cu") else []
        cmd = [NVCC, *ARCH, *common, *lang, "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    for o in objs:
        os.remove(o)
    # the drop-in executables: the reference's main() on DEMClumpMain, and
    # the sphere-only drivers on DEMmain
    for name, srcs in (("nbody_clump_b200", ["main.cpp", "dem_clump_main.cpp"]),
                       ("nbody_sphere_b200", ["sphere_main.cpp", "dem_main.cpp"])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(HERE), "include"),
               *[os.path.join(CSRC, f) for f in srcs], "-L", HERE, "-lnbc", "-Wl,-rpath,$ORIGIN",
               "-o", os.path.join(HERE, name)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"drop-in executable {name} failed to link")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
