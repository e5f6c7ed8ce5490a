"""Build recipe for the oracle (test infrastructure only).

Compiles the FP64 CPU restatement into oracle/_build/liboracle.so with
g++ in ISO C++ mode and -ffp-contract=off, so that floating-point operations
follow the written order (the reference's own CMAKE_CXX_EXTENSIONS OFF mode).
The reference itself cannot be compiled here (Eigen, Boost, oneTBB and ddx
are absent and it needs GCC >= 14), so there is no oracle/_ref build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SOURCES = [os.path.join(HERE, "oracle.cpp")]
HEADERS = [os.path.join(HERE, "oracle_core.hpp"),
           os.path.join(HERE, "..", "include", "forcesmith_gpu.h")]


def build(force=False, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(p) for p in SOURCES + HEADERS)
        if os.path.getmtime(LIB) >= newest:
            return LIB
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-fopenmp",
           "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
           "-Wno-unused-parameter", *SOURCES, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
