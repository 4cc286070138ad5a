"""Builds simcore_b200/libsimcore_b200.so (the C-ABI of include/simcore_gpu.h)
in-tree with nvcc for sm_100a.

Every CUDA unit is compiled with --fmad=false: the FP64 stages reproduce the
reference's contraction-free arithmetic bit for bit; FP32 code issues its
fused multiply-adds explicitly.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsimcore_b200.so")
BUILD_DIR = os.path.join(ROOT, "_build")

CU_SOURCES = ["sc_kernels.cu", "sc_kernels_fast.cu", "sc_api.cu", "sc_graph.cu", "sc_autotune.cu",
              "sc_state.cu", "sc_output.cu", "sc_analysis.cu", "sc_xlinks.cu", "sc_noalloc.cu",
              "sc_insert_gpu.cu", "sc_rebuild.cu"]
# Units compiled with FMA contraction (everything else keeps --fmad=false).
FMAD_SOURCES = {"sc_kernels_fast.cu"}
CPP_SOURCES = ["sc_insert.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in ("nvcc", "/usr/local/cuda/bin/nvcc"):
        if shutil.which(c):
            return shutil.which(c)
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_verbose=False):
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
               if f.endswith((".h", ".cuh"))] + [os.path.join(ROOT, "include", "simcore_gpu.h")]
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo"]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            fmad = "--fmad=true" if src in FMAD_SOURCES else "--fmad=false"
            cmd = [nvcc] + ARCH + common + [fmad] + inc + ["-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc] + ARCH + common + inc + ["-x", "c++", "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv,
                ptxas_verbose="--ptxas" in sys.argv))
