"""Build the chainamps_b200 CUDA library in-tree (nvcc, sm_100a).

    python -m chainamps_b200.build        # -> chainamps_b200/libchainamps_b200.so

The shared library is the product: every kernel is compiled for sm_100a
(B200) only, and the C ABI is declared in include/chainamps_b200.h.

Each source compiles to its own object under _build/ (in parallel), then
nvcc links the library.  A stamp file beside the library records the
SHA-256 of every source, header and flag that went into it; the library is
rebuilt whenever that digest differs, so a library built from other sources
is never reused because its modification time happens to be newer.
"""
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchainamps_b200.so")
STAMP = LIB + ".sha256"
OBJDIR = os.path.join(ROOT, "_build", "chainamps_b200")
SOURCES = ["capi.cu", "heff.cu", "kernels.cu", "zgemm_fp64.cu", "svd.cu", "split_tf32.cu", "tc_gemm.cu", "noalloc.cu",
           "dmrg.cu", "adjoint.cu", "unitcell.cu", "mpxio.cu", "canonical.cu", "canonical_tc.cu", "cgemm_fp32.cu",
           "projector.cu"]
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
LIBS = ["-lcusolver", "-lcublas"]


def sources():
    missing = [s for s in SOURCES if not os.path.exists(os.path.join(CSRC, s))]
    if missing:
        raise FileNotFoundError(f"missing CUDA sources: {missing}")
    return list(SOURCES)


def _inputs():
    files = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".h", ".cuh")))
    files.append(os.path.join(ROOT, "include", "chainamps_b200.h"))
    return files


def digest(extra=()):
    h = hashlib.sha256()
    for f in _inputs():
        h.update(os.path.relpath(f, ROOT).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(ARCH + CFLAGS + LIBS + list(extra) + sources()).encode())
    return h.hexdigest()


def nvcc_compile(src, extra=()):
    obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
    cmd = [os.path.join(CUDA, "bin", "nvcc"), *ARCH, *CFLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    return cmd, obj


def nvcc_link(objs, out=LIB):
    return [os.path.join(CUDA, "bin", "nvcc"), *ARCH, "-shared", *objs, "-o", out, "-L",
            os.path.join(CUDA, "lib64"), *LIBS, "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]


def up_to_date(extra=()):
    if not os.path.exists(LIB) or not os.path.exists(STAMP):
        return False
    with open(STAMP) as fh:
        return fh.read().strip() == digest(extra)


def build(verbose=False, extra=(), force=False):
    if not force and up_to_date(extra):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = [nvcc_compile(s, extra) for s in sources()]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        futs = {ex.submit(subprocess.run, cmd, capture_output=True, text=True): cmd for cmd, _ in jobs}
        for fut in cf.as_completed(futs):
            r = fut.result()
            if verbose:
                print(" ".join(futs[fut]), flush=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, futs[fut])
    cmd = nvcc_link([o for _, o in jobs])
    if verbose:
        print(" ".join(cmd), flush=True)
    if os.path.exists(STAMP):
        os.remove(STAMP)
    subprocess.run(cmd, check=True)
    with open(STAMP, "w") as fh:
        fh.write(digest(extra) + "\n")
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
    print(LIB)
