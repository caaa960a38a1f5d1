"""Build the native library libcvtpm.so in-tree (cvt_b200/libcvtpm.so).

Device code is compiled for sm_100a only.  -fmad=false keeps nvcc from fusing
a*b+c on its own: the kernels place every fused multiply-add explicitly, so
their arithmetic is fixed by the source.  Host code is built with
-ffp-contract=off for the same reason.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcvtpm.so")
BUILD = os.path.join(HERE, "_build")

CU_SOURCES = ["pm_kernels.cu", "pm_propagate.cu", "pm_api.cu", "pm_vpm.cu", "pm_svpm.cu", "pm_learn.cu"]
CXX_SOURCES = ["pm_scene.cpp", "pm_io.cpp"]
HEADERS = ["pm_math.cuh", "pm_device.cuh", "pm_window.cuh", "pm_kernels.h"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include")]


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


def build(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES + CXX_SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "cvtpm.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    nvcc = _nvcc()
    for f in CU_SOURCES:
        o = os.path.join(BUILD, f + ".o")
        cmd = [nvcc] + NVCC_FLAGS + ["-c", os.path.join(CSRC, f), "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(o)
    for f in CXX_SOURCES:
        o = os.path.join(BUILD, f + ".o")
        subprocess.run(["g++", "-O2", "-fPIC", "-ffp-contract=off", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                        "-c", os.path.join(CSRC, f), "-o", o], check=True)
        objs.append(o)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, "-Wno-deprecated-gpu-targets", "-shared", "-o", tmp] + objs + ["-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="-f" in sys.argv, verbose="-v" in sys.argv))
