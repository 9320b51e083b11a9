"""Builds libhrrt_gpu.so in-tree (sm_100a) with nvcc.

The CUDA sources are compiled with -fmad=false: the reference projector is an
x86-64 SSE2 build that never fuses multiply and add, and the kernels keep its
expression order, so their results are bit-identical where the algorithm is.
Host code (geometry tables) is compiled with -ffp-contract=off for the same
reason.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhrrt_gpu.so")
CLI = os.path.join(HERE, "hrrt_osem3d_gpu")
LMCLI = os.path.join(HERE, "lmhistogram_gpu")

SOURCES = ["kernels.cu", "hrrt_gpu.cu", "batch.cu", "geometry.cpp", "listmode.cu", "lm_tables.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_library(force=False, verbose=False):
    """Compile every source to an object under _build/ (in parallel), then
    link libhrrt_gpu.so."""
    from concurrent.futures import ThreadPoolExecutor
    deps = [os.path.join(CSRC, s) for s in SOURCES]
    deps += [os.path.join(CSRC, h) for h in ("kernels.cuh", "geometry.h", "lm_tables.h", "context.h")]
    deps += [os.path.join(ROOT, "include", "hrrt_gpu.h"), __file__]
    if not force and _newer(LIB, deps):
        return LIB
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
             "-I" + os.path.join(ROOT, "include")]
    if verbose:
        flags.insert(0, "-Xptxas=-v")

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        r = subprocess.run([nvcc(), *flags, "-c", os.path.join(CSRC, src), "-o", obj], capture_output=True, text=True)
        return obj, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for obj, r in results:
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        if verbose:
            sys.stderr.write(r.stderr)
    r = subprocess.run([nvcc(), *ARCH, "--shared", "-o", LIB + ".tmp"] + [o for o, _ in results] + ["-lcudart"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def _build_tool(name, force):
    src = os.path.join(CSRC, "cli", name + ".cpp")
    exe = os.path.join(HERE, name)
    if not os.path.exists(src):
        return None
    deps = [src, LIB, os.path.join(ROOT, "include", "hrrt_gpu.h")]
    if not force and _newer(exe, deps):
        return exe
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include"), src,
           "-o", exe + ".tmp", "-L" + HERE, "-lhrrt_gpu", "-Wl,-rpath,$ORIGIN", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n" + r.stdout + r.stderr)
    os.replace(exe + ".tmp", exe)
    return exe


def build_cli(force=False):
    """The command lines: hrrt_osem3d_gpu (returned) and lmhistogram_gpu."""
    _build_tool("lmhistogram_gpu", force)
    return _build_tool("hrrt_osem3d_gpu", force)


def build_lmhistogram(force=False):
    return _build_tool("lmhistogram_gpu", force)


def build_all(force=False, verbose=False):
    build_library(force=force, verbose=verbose)
    build_cli(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
