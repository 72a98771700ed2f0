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


def local_deps(path, seen=None):
    """The files `path` includes by a quoted #include that resolve in csrc/ or include/, recursively."""
    import re
    seen = set() if seen is None else seen
    with open(path) as f:
        names = re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read(), re.M)
    for name in names:
        for d in (os.path.dirname(path), os.path.join(HERE, "csrc"), os.path.join(os.path.dirname(HERE), "include")):
            q = os.path.normpath(os.path.join(d, name))
            if os.path.exists(q):
                if q not in seen:
                    seen.add(q)
                    local_deps(q, seen)
                break
    return seen


def obj_of(src):
    return os.path.join(LIB_DIR, "obj", os.path.basename(src) + ".o")


def stale(src, obj):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(f) > t for f in [src, __file__] + sorted(local_deps(src)))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force=False, verbose=False, ptxas_info=False, jobs=None):
    """Compiles the sources whose object is older than the source or one of its local includes (all
    of them with force), in parallel, and links the library."""
    from concurrent.futures import ThreadPoolExecutor
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.join(LIB_DIR, "obj"), exist_ok=True)
    todo = [s for s in sources() if force or ptxas_info or stale(s, obj_of(s))]

    def compile_one(src):
        cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj_of(src)]
        return src, subprocess.run(cmd, capture_output=True, text=True)

    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(compile_one, todo))
    failed = []
    for src, r in results:
        if verbose or r.returncode != 0 or ptxas_info:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + [obj_of(s) for s in sources()] + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
