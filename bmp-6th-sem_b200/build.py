"""Builds libpicb200.so in-tree for sm_100a (nvcc, no GPU needed).

    python bmp-6th-sem_b200/build.py [--debug]

The library is plain CUDA C++ behind the C ABI in include/pic_capi.h and
include/sycl_pic_compat.h; it does not link against PyTorch.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpicb200.so")
SOURCES = ["context.cu", "particles.cu", "poisson.cu", "compat.cu", "picdat.cu", "noalloc.cu", "warmstart.cu", "ensemble.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def build(debug: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, "pic_internal.h"),
                                                          os.path.join(ROOT, "include", "pic_capi.h")])
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= newest and not debug:
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
                    "-I", os.path.join(ROOT, "include"), "-I", CSRC, "--expt-relaxed-constexpr",
                    "-ccbin", "g++"]
    if debug:
        flags += ["-DPIC_DEBUG=1"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        subprocess.run(["nvcc", *flags, "-c", s, "-o", o], check=True)
        objs.append(o)
    tmp = OUT + ".tmp"
    subprocess.run(["nvcc", *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-ccbin", "g++"],
                   check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, verbose="-v" in sys.argv))
