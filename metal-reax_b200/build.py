"""Builds librxcuda.so (the C-ABI engine) in-tree for sm_100a with nvcc.

    python metal-reax_b200/build.py [--verbose]

Every translation unit is compiled separately (parallel) into _build/ and linked into metal-reax_b200/librxcuda.so.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
SRC = PKG / "csrc"
OUT = PKG / "librxcuda.so"
BUILD = REPO / "_build"
SOURCES = ["engine.cu", "kernels_nb.cu", "kernels_bonded.cu", "md_kernels.cu", "ffield.cpp", "noalloc.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I" + str(REPO / "include")]


def _compile(src, verbose):
    obj = BUILD / (src + ".o")
    srcp = SRC / src
    deps = [srcp] + list(SRC.glob("*.hpp")) + list(SRC.glob("*.cuh")) + [REPO / "include" / "rxcuda.h"]
    if obj.exists() and all(obj.stat().st_mtime >= p.stat().st_mtime for p in deps):
        return obj
    cmd = [NVCC] + ARCH + FLAGS + ["-c", str(srcp), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    if verbose and r.stderr:
        print(r.stderr, flush=True)
    return obj


LAMMPS_SRC = [PKG / "lammps" / "rx_lammps.cpp", PKG / "lammps" / "rx_lammps_capi.cpp"]
LAMMPS_OUT = PKG / "librxlammps.so"


def build_lammps_bridge():
    """librxlammps.so: the LAMMPS-side bridge of the CUDA backend (plain C++ over librxcuda.so's C ABI)."""
    deps = LAMMPS_SRC + [PKG / "lammps" / "rx_lammps.hpp", REPO / "include" / "rxcuda.h", OUT]
    if LAMMPS_OUT.exists() and all(LAMMPS_OUT.stat().st_mtime >= p.stat().st_mtime for p in deps):
        return LAMMPS_OUT
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", str(LAMMPS_OUT)] + [str(p) for p in LAMMPS_SRC] + \
          ["-L" + str(PKG), "-lrxcuda", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("bridge build failed:\n%s%s" % (r.stdout, r.stderr))
    return LAMMPS_OUT


def build(verbose=False):
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if not (OUT.exists() and all(OUT.stat().st_mtime >= o.stat().st_mtime for o in objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(OUT)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    build_lammps_bridge()
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
