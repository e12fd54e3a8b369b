"""Build libpcg.so, the CUDA library behind include/pcg.h, for sm_100a.

Usage: python -m picopic_b200.build [--force]

Each translation unit is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``picopic_b200/_build`` and
linked into ``picopic_b200/libpcg.so`` (CUDA runtime linked statically, so
the library only needs the driver).  The double-precision particle kernels
are compiled with ``--fmad=false``: they follow the reference operation
order and must not be contracted into FMAs.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libpcg.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(REPO, "include"),
          "-I" + CSRC, "--expt-relaxed-constexpr"]
UNITS = {
    "pcg_api.cu": [],
    "pcg_util.cu": [],
    "pcg_kernels_f64.cu": ["--fmad=false"],
    # the float production path: approximate division/sqrt (2 ulp) and FTZ
    "pcg_kernels_f32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "pcg_init.cu": [],
    "pcg_noalloc.cu": ["--fmad=false"],
    "pcg_diag.cu": ["--fmad=false"],
    "pcg_collide.cu": ["--fmad=false"],
    "pcg_collide_crowded.cu": ["--fmad=false"],
    "pcg_mlp.cu": [],
    "pcg_learned.cu": ["--fmad=false"],
    "pcg_maps.cu": ["--fmad=false"],
    "pcg_ensemble.cu": [],
    "pcg_region.cu": ["--fmad=false"],
}


def _deps(unit):
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith((".cuh", ".h"))] + [os.path.join(CSRC, unit), os.path.join(REPO, "include", "pcg.h")]


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        newest = max(os.path.getmtime(d) for d in _deps(unit))
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
            continue
        cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        subprocess.check_call([NVCC, *ARCH, "-shared", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
