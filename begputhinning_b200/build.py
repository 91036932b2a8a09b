"""Build the native libraries in-tree.

``libbgt.so``       CUDA kernels (sm_100a) + C ABI + drop-in C++ entry points
``libbgt_synth.so`` seeded synthetic workload generators (host C++)

Run ``python -m begputhinning_b200.build`` (or ``build()``).  nvcc cross-compiles
for sm_100a without a GPU.  Objects go to ``_build/`` (not committed); the
shared libraries land next to this file so they travel with the package.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["kernels.cu", "resident.cu", "host.cu", "segments.cu", "centerline.cu", "noalloc.cu", "serve.cu"]
CXX_SOURCES = ["dropin.cpp"]
HEADERS = ["common.cuh", "rules.cuh", "tiles.cuh", "kernels.cuh", "host.h"]

LIB = os.path.join(PKG, "libbgt.so")
SYNTH = os.path.join(PKG, "libbgt_synth.so")


def _digest(paths):
    h = hashlib.sha256()
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    return h.hexdigest()


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd[:3])} ...")
    return r.stdout + r.stderr


def _inputs():
    srcs = [os.path.join(CSRC, f) for f in CU_SOURCES + CXX_SOURCES + HEADERS]
    srcs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return srcs


def build_lib(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    """Compile libbgt.so (skipped when sources are unchanged since the last build)."""
    os.makedirs(BUILD, exist_ok=True)
    stamp = os.path.join(BUILD, "libbgt.sha256")
    dig = _digest(_inputs())
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == dig:
        return LIB
    common = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}"]
    objs = []
    log = []
    for f in CU_SOURCES:
        o = os.path.join(BUILD, f + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", *common, "-c", os.path.join(CSRC, f), "-o", o]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        log.append(_run(cmd, verbose))
        objs.append(o)
    for f in CXX_SOURCES:
        o = os.path.join(BUILD, f + ".o")
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}",
               "-I/usr/local/cuda/include", "-c", os.path.join(CSRC, f), "-o", o]
        log.append(_run(cmd, verbose))
        objs.append(o)
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs], verbose)
    os.replace(tmp, LIB)
    with open(stamp, "w") as f:
        f.write(dig)
    if ptxas_info:
        with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
            f.write("\n".join(log))
    return LIB


def build_synth(verbose: bool = False) -> str:
    src = os.path.join(CSRC, "synth.cpp")
    os.makedirs(BUILD, exist_ok=True)
    stamp = os.path.join(BUILD, "synth.sha256")
    dig = _digest([src])
    if os.path.exists(SYNTH) and os.path.exists(stamp) and open(stamp).read() == dig:
        return SYNTH
    tmp = SYNTH + ".tmp"
    _run(["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-o", tmp, src], verbose)
    os.replace(tmp, SYNTH)
    with open(stamp, "w") as f:
        f.write(dig)
    return SYNTH


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> None:
    build_synth(verbose)
    build_lib(verbose, ptxas_info, force)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv, force="--force" in sys.argv)
    print(LIB)
