"""Builds the CUDA library liblbmb200.so in-tree (sm_100a).

Usage: python -m fortran_loadfile_mitiwing_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "liblbmb200.so")
ROOT = os.path.dirname(HERE)

SOURCES = ["lbm_capi.cu", "kf_kernel.cu", "ib_kernels.cu", "host_io.cu", "host_xfer.cu", "residual_device.cu",
           "lbm_batch.cu", "output_io.cu"]
HEADERS = ["lbm_common.cuh", "lbm_internal.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "lbm_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, out=None, defines=()):
    """Compiles every CUDA source into one shared library; returns its path.
    `out` and `defines` (-D values) build a variant elsewhere, for tuning."""
    lib = out or LIB
    if not force and out is None and not _stale():
        return LIB
    libdir = os.path.dirname(lib)
    os.makedirs(libdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(libdir, src.replace(".cu", ".o"))
        cmd = [_nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-I", os.path.join(ROOT, "include"), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", lib,
           "-Xlinker", "--exclude-libs,ALL"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return lib


DRIVER_SRC = os.path.join(CSRC, "lbm_main.cpp")
DRIVER = os.path.join(LIBDIR, "lbm_main")


def build_driver(force=False, verbose=False):
    """Compiles the driver program (main.f90's loop over the C ABI) with the
    host compiler, linked against the library in the same directory."""
    lib = build(force=force, verbose=verbose)
    if not force and os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(
            os.path.getmtime(DRIVER_SRC), os.path.getmtime(lib)):
        return DRIVER
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
           DRIVER_SRC, "-o", DRIVER, "-L", LIBDIR, "-llbmb200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


def build_oracle(verbose=False):
    """Builds the CPU oracle (test infrastructure) with its Makefile."""
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_driver(verbose=True)
