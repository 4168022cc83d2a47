"""Build libpbemcs.so (the sm_100a CUDA library) in the package directory.

    python -m thruster_cx_code_b200._build

Compiles three translation units with nvcc for sm_100a and links them:
  csrc/pb_runtime.cu  the runtime, the C-ABI and (included) the particle and diagnostic
                      kernels, with fused multiply-add contraction disabled: the particle
                      arithmetic reproduces NumPy's separately rounded operations;
  csrc/pb_poisson.cu  the FP32 MG-PCG field solve, with contraction allowed (its result is
                      compared with SuperLU to a tolerance, not bit for bit);
  csrc/pb_mgdev.cu    the multigrid hierarchy rebuilt on the device after cells break
                      (explicitly rounded arithmetic, bit-equal to the host build).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpbemcs.so")
SOURCES = ["pb_runtime.cu", "pb_particles.cu", "pb_poisson.cu", "pb_mgdev.cu", "pb_misc.cu", "pb_batch.cu",
           "pb_common.cuh",
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


UNITS = (("pb_runtime.cu", "false"), ("pb_poisson.cu", "true"), ("pb_mgdev.cu", "false"))


def _run(cmd, verbose):
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libpbemcs.so")
    if verbose:
        sys.stderr.write(r.stderr)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    common = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc")]
    objs = []
    tmp = LIB + ".objs"
    os.makedirs(tmp, exist_ok=True)
    try:
        for src, fmad in UNITS:
            obj = os.path.join(tmp, src.replace(".cu", ".o"))
            contract = "fast" if fmad == "true" else "off"
            _run([nvcc()] + common + [f"-fmad={fmad}", "-Xcompiler", f"-fPIC,-ffp-contract={contract}", "-c",
                                      os.path.join(HERE, "csrc", src), "-o", obj], verbose)
            objs.append(obj)
        _run([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + objs + ["-o", LIB + ".tmp"], False)
    finally:
        for o in objs:
            if os.path.exists(o):
                os.remove(o)
        if os.path.isdir(tmp):
            os.rmdir(tmp)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
