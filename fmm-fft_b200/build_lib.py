"""Builds libfmmfft_b200.so in this directory (in-tree, so it travels with the repository).

    python fmm-fft_b200/build_lib.py          # incremental
    python fmm-fft_b200/build_lib.py --force

CUDA sources are compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a); host
sources are C99 (gcc).  The CUDA runtime is linked statically into the library.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfmmfft_b200.so")
BUILD = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["fmmfft_kernels.cu"]
C_SOURCES = ["fmmfft_ops.c", "fmmfft_api.c", "fmmfft_serve.c"]
HEADERS = ["fmmfft_internal.h", "fmmfft_tc.cuh", os.path.join("..", "..", "include", "fmmfft.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xptxas", "-O3", "--expt-relaxed-constexpr",
]
CC_FLAGS = ["-O2", "-std=gnu99", "-fPIC", "-Wall", "-Wno-unused-function",
            "-I" + os.path.join(CUDA_HOME, "include")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {os.path.basename(cmd[-1])}")
    return r


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", "-o", o, s]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            cmd = ["gcc"] + CC_FLAGS + ["-c", "-o", o, s]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(o)
    if force or _newer(OUT, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + \
              ["-cudart", "static", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
