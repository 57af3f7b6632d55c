"""Build libdvgpu.so in-tree for sm_100a with nvcc.

    python zkp-dynaverse_b200/build.py [--verbose-ptxas]

Compiles every csrc/*.cu into zkp-dynaverse_b200/lib/libdvgpu.so.  Objects
go to zkp-dynaverse_b200/_build/.  Rebuilds only what changed (source or
any csrc header newer than the object).
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("DVGPU_BUILD_DIR", os.path.join(HERE, "_build"))
LIB = os.environ.get("DVGPU_LIB_OUT", os.path.join(HERE, "lib", "libdvgpu.so"))
LIB_DIR = os.path.dirname(LIB)
EXTRA = os.environ.get("DVGPU_EXTRA_FLAGS", "").split()
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]


def _newest_header():
    heads = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(h) for h in heads)


def build(verbose_ptxas=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_time = _newest_header()
    objs, procs = [], []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
            continue
        cmd = [NVCC] + ARCH + FLAGS + EXTRA + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose_ptxas:
            sys.stdout.write(out)
        if p.returncode != 0:
            failed = True
            sys.stdout.write(f"FAILED: {src}\n")
    if failed:
        raise RuntimeError("nvcc failed")
    if procs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv)
    print(LIB)
