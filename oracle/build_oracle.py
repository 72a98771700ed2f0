"""Build recipe for the CPU oracle (test infrastructure only).

Two shared libraries:
  oracle/liboracle.so          the plain-C restatement (pb_oracle.c), built everywhere.
  oracle/_ref/libproto_ref.so  the reference's own header-only C++ compiled from where it lies
                               (ref_driver.cpp), built only where the reference tree is present.
Both are compiled with -ffp-contract=off so that no multiply-add is fused: the oracle's floating
point follows the reference's written operation order exactly.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout's mount point in the build container (read only); PROTO_REFERENCE_ROOT
# points the recipe elsewhere. Where neither exists the reference-built library is skipped.
REF_ROOT = os.environ.get("PROTO_REFERENCE_ROOT", "/root/reference")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(cmd))


def build_port(force=False):
    out = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "pb_oracle.c")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    _run(["gcc", "-O3", "-std=c11", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
          src, "-o", out, "-lm"])
    return out


def build_ref(force=False):
    """Compile the reference headers into oracle/_ref/libproto_ref.so (skipped without them)."""
    inc = os.path.join(REF_ROOT, "include")
    if not os.path.isdir(inc):
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    out = os.path.join(outdir, "libproto_ref.so")
    src = os.path.join(HERE, "ref_driver.cpp")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    _run(["g++", "-std=c++17", "-O3", "-ffp-contract=off", "-fPIC", "-shared",
          "-DDIM=3", "-DPR_TURN_OFF_TIMERS", "-DNDEBUG", "-DPR_DISABLE_INIT_CHECKS",
          "-I" + inc, "-I" + os.path.join(inc, "base"), "-I" + os.path.join(inc, "utils"),
          "-I" + os.path.join(REF_ROOT, "examples", "_common"),
          "-I" + os.path.join(REF_ROOT, "examples", "_archived", "LevelMultigrid", "src"),
          "-w", src, "-o", out])
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_port(force))
    print(build_ref(force))
