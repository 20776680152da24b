"""Build the sm_100a CUDA library in-tree: milkywayathome_client_b200/libnbody_b200.so.

Every translation unit is compiled by nvcc for sm_100a only, with -fmad=false so the FP64
code keeps the reference CPU build's rounding (no FMA contraction); FP32 code that wants a
fused multiply-add spells out fmaf().  The adjoint kernels (nb_adjoint.cu) have no reference
rounding to keep and are compiled with contraction on.

    python -m milkywayathome_client_b200.build [--force] [--verbose]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnbody_b200.so")
SOURCES = ["nb_sort.cu", "nb_tree.cu", "nb_walk.cu", "nb_mixed.cu", "nb_api.cu", "nb_noalloc.cu", "nb_adjoint.cu", "nb_batch.cu", "nb_ic.cu", "nb_likelihood.cu", "nb_lmc.cu"]
HEADERS = ["nb_common.cuh", "nb_potential.cuh", "nb_tree_util.cuh", "nb_crmath.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-Xptxas", "-v"]
FMAD_ON = {"nb_adjoint.cu"}          # everything else: -fmad=false (reference rounding)


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    inc = os.path.join(os.path.dirname(HERE), "include")
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(inc, "nbody_b200.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            fmad = ["-fmad=true"] if src in FMAD_ON else ["-fmad=false"]
            cmd = [NVCC] + ARCH + FLAGS + fmad + ["-I", inc, "-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            log = os.path.join(BUILD, src.replace(".cu", ".ptxas.txt"))
            with open(log, "w") as f:
                f.write(r.stdout + r.stderr)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed for %s" % src)
            if verbose:
                sys.stderr.write(r.stderr)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libnbody_b200.so failed")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
