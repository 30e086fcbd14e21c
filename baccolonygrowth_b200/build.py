"""Build of the sm_100a shared library (libbcg.so) from csrc/.

The library is compiled in-tree with nvcc for sm_100a only.  The mechanics
and field kernels are built with -fmad=false so that their products and
sums round like the reference's x86-64 build (no FMA contraction).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbcg.so")

CU_SOURCES = ["ctx.cu", "mech.cu", "fields.cu", "mg.cu", "mg_smooth.cu", "nutrients.cu", "steady.cu", "output.cu"]
CPP_SOURCES = ["host.cpp", "sim.cpp", "writer.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fno-fast-math", "--expt-relaxed-constexpr"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    """Compile csrc/ into baccolonygrowth_b200/libbcg.so (sm_100a)."""
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "bcg.h"))
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [sp] + headers):
            continue
        if src.endswith(".cu"):
            cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-c", sp, "-o", obj]
        else:
            cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-x", "c++", "-c", sp, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
