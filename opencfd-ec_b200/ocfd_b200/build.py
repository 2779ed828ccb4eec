"""Builds libocfd_b200.so in-tree with nvcc for sm_100a.

The FP64 translation units (setup.cu, solver_fp64.cu) are compiled with --fmad=false so every
a*b+c is rounded twice, as the FP64 reference evaluates it; the mixed-precision unit keeps FMA and
the IEEE-rounded FP32 division and square root (the approximate ones made the mixed step 8 % faster
and its residual norms leave the stated 1e-3 tolerance against FP64 after 10 steps).
"""
import os
import subprocess
import sys

from . import ROOT_DIR

CSRC = os.path.join(ROOT_DIR, "csrc")
LIB_PATH = os.path.join(ROOT_DIR, "libocfd_b200.so")
BUILD_DIR = os.path.join(ROOT_DIR, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]

UNITS = [
    ("setup.cu", ["--fmad=false"]),
    ("solver_fp64.cu", ["--fmad=false"]),
    ("solver_mixed.cu", []),
    ("capi.cu", []),
]


def sources():
    """Everything the library depends on, this file (its compiler flags) included."""
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h", ".inc"))] + [
        os.path.join(os.path.dirname(ROOT_DIR), "include", "ocfd_ec_gpu.h"), os.path.abspath(__file__)]


def up_to_date():
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(s) <= t for s in sources())


DRIVER_SRC = os.path.join(ROOT_DIR, "driver", "ocfd_drive.cpp")
DRIVER_PATH = os.path.join(ROOT_DIR, "ocfd_drive")


def build_driver(force=False):
    """The compiled C++ caller of the C-ABI (driver/ocfd_drive.cpp), linked against the in-tree
    library (found next to it at run time)."""
    deps = [DRIVER_SRC, LIB_PATH, os.path.join(os.path.dirname(ROOT_DIR), "include", "ocfd_ec_gpu.h")]
    if not force and os.path.exists(DRIVER_PATH) and all(os.path.getmtime(d) <= os.path.getmtime(DRIVER_PATH) for d in deps):
        return DRIVER_PATH
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-ffp-contract=off", "-std=c++17", DRIVER_SRC, "-L" + ROOT_DIR, "-locfd_b200",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER_PATH + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(DRIVER_PATH + ".tmp", DRIVER_PATH)
    return DRIVER_PATH


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        build_driver()
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    procs = []
    for src, flags in UNITS:
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        cmd = [NVCC] + ARCH + COMMON + list(flags) + list(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"), file=sys.stderr)
    if failed:
        msg = "\n".join("---- %s\n%s" % f for f in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    tmp = LIB_PATH + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    build_driver(force=True)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB_PATH)
