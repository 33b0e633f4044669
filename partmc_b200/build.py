"""Build libpmc_coag_gpu.so in-tree with nvcc for sm_100a.

The replay translation unit is compiled with -fmad=false so that its FP64
arithmetic rounds every multiply and add separately, as the reference's
gfortran build does.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpmc_coag_gpu.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"] + ARCH

UNITS = [
    ("pmc_coag.cu", []),
    ("pmc_replay.cu", ["-fmad=false"]),
    ("pmc_noalloc.cu", []),
]
HEADERS = ["pmc_physics.cuh", "pmc_state.cuh", "pmc_kernels.cuh", "pmc_merge.cuh", "pmc_particle.cuh",
           "pmc_replay.cuh", "pmc_sample.cuh"]


def _nvcc():
    for cand in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"]:
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "pmc_coag_gpu.h")]
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [_nvcc()] + COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
