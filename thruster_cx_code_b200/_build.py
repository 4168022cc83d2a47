"""Build libpbemcs.so (the sm_100a CUDA library) in the package directory.

    python -m thruster_cx_code_b200._build

Compiles csrc/pb_runtime.cu (a unity build that includes the kernel sources) with nvcc
for sm_100a.  Fused multiply-add contraction is disabled for the whole library: the
particle arithmetic reproduces NumPy's separately rounded operations.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpbemcs.so")
SOURCES = ["pb_runtime.cu", "pb_particles.cu", "pb_poisson.cu", "pb_misc.cu", "pb_batch.cu", "pb_common.cuh",
           "pb_kernels.cuh", "pb_misc.cuh", "pb_poisson.cuh", "pb_mg_host.hpp"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, "csrc", f) for f in SOURCES] + [os.path.join(ROOT, "include", "pbemcs.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc"),
           os.path.join(HERE, "csrc", "pb_runtime.cu"), "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libpbemcs.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
