"""Builds libct.so (the C ABI of include/ct.h) for sm_100a, in tree.

    python cube-tracing_b200/build.py

The library is compiled with --fmad=false -prec-div=true -prec-sqrt=true:
multiply-adds are never contracted implicitly and divisions / square roots
are IEEE round-to-nearest, so results follow the operation order written in
the kernels (see csrc/ct_math.cuh).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = ["ct_api.cu", "ct_accel.cu", "ct_kernels.cu", "ct_noalloc.cu", "ct_nrc.cu", "ct_profile.cu", "ct_state.cu"]
OUT = os.path.join(HERE, "cube_tracing", "libct.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
         "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC,-O2", "-I", os.path.join(ROOT, "include"),
         "-I", os.path.join(HERE, "csrc")]


HOST_SRC = ["ct_host.cpp", "ct_host_check.cpp"]
HOST_OUT = os.path.join(HERE, "host", "ct_host_check")


def build_host(verbose=False):
    """The C++ host side (host/ct_host.cpp, ct::Renderer) and its check
    program, linked against libct.so."""
    srcs = [os.path.join(HERE, "host", s) for s in HOST_SRC]
    deps = srcs + [os.path.join(HERE, "host", "ct_host.hpp"), os.path.join(ROOT, "include", "ct.h"), OUT]
    if os.path.exists(HOST_OUT) and os.path.getmtime(HOST_OUT) >= max(os.path.getmtime(p) for p in deps):
        return HOST_OUT
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(HERE, "host"),
           "-o", HOST_OUT] + srcs + ["-L", os.path.dirname(OUT), "-lct", "-Xlinker", "-rpath,$ORIGIN/../cube_tracing"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return HOST_OUT


def build(verbose=False, extra=()):
    srcs = [os.path.join(HERE, "csrc", s) for s in SRC]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(ROOT, "include", "ct.h")] +
                 [os.path.join(HERE, "csrc", h) for h in os.listdir(os.path.join(HERE, "csrc"))
                  if h.endswith((".cuh", ".h"))])
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= newest and not extra:
        return OUT
    cmd = [NVCC, "-shared", "-o", OUT] + FLAGS + list(extra) + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(verbose=True, extra=extra))
    print(build_host(verbose=True))
