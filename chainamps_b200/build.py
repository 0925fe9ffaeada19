"""Build the chainamps_b200 CUDA library in-tree (nvcc, sm_100a).

    python -m chainamps_b200.build        # -> chainamps_b200/libchainamps_b200.so

The shared library is the product: every kernel is compiled for sm_100a
(B200) only, and the C ABI is declared in include/chainamps_b200.h.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchainamps_b200.so")
SOURCES = ["capi.cu", "heff.cu", "kernels.cu", "zgemm_fp64.cu", "svd.cu", "split_tf32.cu", "tc_gemm.cu", "noalloc.cu", "dmrg.cu", "adjoint.cu", "unitcell.cu", "mpxio.cu"]
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def nvcc_cmd(out=LIB, extra=()):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    return [os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
            "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
            *extra, *srcs, "-o", out, "-L", os.path.join(CUDA, "lib64"), "-lcusolver", "-lcublas",
            "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]


def build(verbose=False, extra=()):
    newest = max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC))
    newest = max(newest, os.path.getmtime(os.path.join(ROOT, "include", "chainamps_b200.h")))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest and not extra:
        return LIB
    cmd = nvcc_cmd(extra=extra)
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
    print(LIB)
