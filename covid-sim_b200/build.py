"""Build the sm_100a sweep library in place: covid-sim_b200/lib/libcovidsim_b200.so.

Usage: python covid-sim_b200/build.py [--force]

The library is one shared object with a C ABI (include/covidsim_b200.h); it
statically links the CUDA runtime so it loads on any host of this image, with or
without a GPU.  Device code is compiled with --fmad=false: every floating-point
expression rounds as written, which keeps results independent of contraction
choices the compiler would otherwise make.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcovidsim_b200.so")

SOURCES = ["cs_sweep.cu", "cs_surrogate.cu", "cs_setup.cu", "cs_host.cpp"]
HEADERS = ["cs_device.cuh", "cs_state.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "covidsim_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs() if os.path.exists(f))


def build(force=False, verbose=False):
    """Compile the library unless it is newer than every input; returns its path."""
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-ccbin", "/usr/bin/g++",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           *[os.path.join(CSRC, f) for f in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
