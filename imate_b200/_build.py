"""Build of the engine library ``imate_b200/libslq_b200.so`` (sm_100a).

One nvcc invocation compiles the CUDA driver/kernels and the host C++ parts
into an in-tree shared library that the Python host loads with ctypes.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libslq_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["slq_engine.cu", "slq_mlp.cu", "slq_rng.cpp", "slq_stats.cpp",
           "slq_order.cpp"]
HEADERS = ["slq_kernels.cuh", "slq_blk.cuh", "slq_rng.h", "slq_tc.cuh"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or \
        "/usr/local/cuda/bin/nvcc"
    return cand


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(INCLUDE, "slq.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, ptxas_info=False):
    """Compile the engine if any source is newer than the library."""
    if not force and not _stale():
        return LIB
    cmd = [nvcc_path(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17",
           "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
           "-ccbin", "/usr/bin/g++", "-shared", "-I" + INCLUDE,
           "-o", LIB + ".tmp"]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          ptxas_info="--ptxas" in sys.argv)
