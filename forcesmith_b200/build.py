"""Build recipe for the in-tree native libraries (sm_100a).

libforcesmith_b200.so  — the CUDA kernels + C ABI (include/forcesmith_gpu.h)
libfs_synth.so         — seeded synthetic configurations (host C++)

Both are compiled in place so that they travel with the source tree.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
GPU_LIB = os.path.join(HERE, "libforcesmith_b200.so")
SYNTH_LIB = os.path.join(HERE, "libfs_synth.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_synth(force=False):
    src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(SYNTH_LIB, [src]):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", src, "-o",
                        SYNTH_LIB + ".tmp"], check=True)
        os.replace(SYNTH_LIB + ".tmp", SYNTH_LIB)
    return SYNTH_LIB


def gpu_sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def build_gpu(force=False, verbose=False, extra=()):
    srcs = gpu_sources()
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INC, "*.h"))
    if not (force or _stale(GPU_LIB, deps)):
        return GPU_LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [d for d in deps if not d.endswith(".cu")]
    objs, jobs = [], []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-I", INC, "-I", CSRC, "--expt-relaxed-constexpr", "-rdc=false",
                   *extra, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append(cmd)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [NVCC, *ARCH, "-shared", *objs, "-o", GPU_LIB + ".tmp", "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(GPU_LIB + ".tmp", GPU_LIB)
    return GPU_LIB


def build(force=False, verbose=False):
    build_synth(force)
    if gpu_sources():
        build_gpu(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
