"""Compile the CUDA backend for sm_100a into bowshock_b200/_lib/libbowshock_b200.so (in-tree, so it travels with the
repository snapshot). Usage: python -m bowshock_b200.build [--verbose]"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libbowshock_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "capi.cu"), os.path.join(HERE, "csrc", "net.cu"), os.path.join(HERE, "csrc", "mesher_dev.cu")]
# translation units compiled without multiply-add contraction (their FP64 arithmetic rounds like the host code it mirrors)
NO_FMAD = {"mesher_dev.cu"}
HEADERS = ["mesher_dev.h", "arena.cuh", "tma.cuh", "stream_copy.cuh", "device_math.cuh", "viscous.cuh", "turbulence.cuh", "host_arena.cuh", "fv_kernels.cu", "forces.cuh", "mesher.cuh", "runner.cuh", "euler3.cuh", "host3.cuh"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(src=None):
    fmad = "-fmad=false" if src is not None and os.path.basename(src) in NO_FMAD else "-fmad=true"
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
            "-I" + os.path.join(ROOT, "include"), fmad, "-Xptxas", "-warn-spills"]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [s for s in SOURCES if os.path.exists(s)] + [os.path.join(HERE, "csrc", h) for h in HEADERS]
    deps.append(os.path.join(ROOT, "include", "bowshock_b200.h"))
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    if not force and not stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(s)]
    # one object per translation unit (each with its own contraction flag), compiled in parallel, then linked
    objs = [os.path.join(LIB_DIR, os.path.basename(s) + ".o") for s in srcs]
    procs = [subprocess.Popen([nvcc()] + flags(s) + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", o, s], stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for s, o in zip(srcs, objs)]
    for s, p in zip(srcs, procs):
        out, errs = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n" + errs[-8000:])
        if verbose:
            print(errs)
    r = subprocess.run([nvcc()] + flags() + ["-shared", "-o", LIB + ".tmp"] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stderr[-8000:])
    for o in objs:
        os.remove(o)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
