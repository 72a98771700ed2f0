"""Build recipe for the sm_100a shared library proto_b200/lib/libproto_b200.so.

nvcc compiles every csrc/*.cu for compute_100a/sm_100a (no other architecture) and links them into
one C-ABI shared library (include/proto_b200.h). The library depends only on the CUDA runtime;
TMA descriptors are encoded through the driver entry point fetched at run time.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libproto_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# host code never contracts a*b+c into FMA (the direct coarse solve's inverse must match the oracle's)
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=default", "-Xcompiler", "-ffp-contract=off"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
        os.path.join(os.path.dirname(HERE), "include", "proto_b200.h")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force=False, verbose=False, ptxas_info=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.join(LIB_DIR, "obj"), exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(LIB_DIR, "obj", os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0 or ptxas_info:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on " + src)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
