"""Build recipe of the C++ adapter test program: g++ against the in-tree
libforcesmith_b200.so and the headers in include/ (forcesmith_gpu.h,
forcesmith_gpu_adapter.hpp, forcesmith_shim.hpp)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIBDIR = os.path.join(ROOT, "forcesmith_b200")
EXE = os.path.join(HERE, "_build", "adapter_test")


def build():
    src = os.path.join(HERE, "adapter_test.cpp")
    deps = [src] + [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    if os.path.exists(EXE) and all(os.path.getmtime(d) <= os.path.getmtime(EXE) for d in deps):
        return EXE
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-pthread", "-I", os.path.join(ROOT, "include"),
           src, "-o", EXE + ".tmp", "-L", LIBDIR, "-lforcesmith_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True)
    os.replace(EXE + ".tmp", EXE)
    return EXE


if __name__ == "__main__":
    print(build())
    sys.exit(0)
