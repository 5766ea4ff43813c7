"""Builds the CUDA engine: one shared library for sm_100a.

    python build.py            # -> _lib/libd3force_b200.so

Every source is compiled with -fmad=false -prec-div=true -prec-sqrt=true
-ftz=false: exact mode reproduces d3-force's f64 arithmetic bit for bit. The
fast mode's precision forms, the network and batched mode (fmm_tc.cu,
mlp.cu, batch.cu) are measured against an FP64 direct sum instead: they are
compiled with FMA contraction on and the fast FP32 division and square root
(FP64 arithmetic is IEEE either way).
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "libd3force_b200.so")
SOURCES = ["engine.cu", "tree.cu", "scan_sort.cu", "forces.cu", "fast.cu", "fmm.cu", "collide_spec.cu", "noalloc.cu",
           "peaks.cu", "fmm_tc.cu", "mlp.cu", "batch.cu"]
# The precision forms are judged by their error against an FP64 direct sum,
# not bit for bit: their translation unit may contract to FMA.
FAST = ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
PER_SOURCE = {"fmm_tc.cu": FAST, "mlp.cu": FAST, "batch.cu": FAST}
EXACT = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]


def build(verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".cuh")]
        deps.append(os.path.join(HERE, "..", "include", "d3force_b200.h"))
        if not os.path.exists(obj) or any(os.path.getmtime(d) > os.path.getmtime(obj) for d in deps):
            cmd = [NVCC] + FLAGS + PER_SOURCE.get(src, EXACT) + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
        objs.append(obj)
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-q" not in sys.argv))
