"""Build libexotx.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python -m exoplasim_b200.build          # incremental
    python -m exoplasim_b200.build --force  # rebuild everything

Objects go to exoplasim_b200/_build/, the library to exoplasim_b200/lib/.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libexotx.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
# per-file extra flags: the plan builder keeps every FP64 product and sum
# separately rounded, in the reference's evaluation order
EXTRA = {"plan.cu": ["-fmad=false"], "radiation_fp64.cu": ["-fmad=false"], "rawout.cu": ["-fmad=false"], "gridpoint_fp64.cu": ["-fmad=false"], "spectral_fp64.cu": ["-fmad=false"]}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _newer(src_paths, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src_paths)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    objs = []
    nv = nvcc()
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    for f in sources():
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f[:-3] + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            cmd = [nv, "-c", src, "-o", obj, "-ccbin", "/usr/bin/g++"] + ARCH + COMMON + EXTRA.get(f, [])
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd, env=env)
    if force or _newer(objs, LIB):
        cmd = [nv, "-shared", "-o", LIB, "-ccbin", "/usr/bin/g++"] + ARCH + objs + ["-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, env=env)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
