"""Build recipe of the CUDA library libdcm_b200.so (sm_100a only).

Compiles every csrc/*.cu with nvcc into one shared object next to this file.
The result is the C-ABI declared in include/dcm.h; nothing here depends on
PyTorch.  Usage:  python build.py [--force]
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdcm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-I" + os.path.join(ROOT, "include"), "-cudart", "static"]
# Kernel files with FP32 instantiations (used only by the mixed-precision
# form): single-precision division as reciprocal-multiply (within 2 ulp)
# instead of the IEEE sequence.  The flag does not touch FP64 division, so
# the FP64 parity path keeps the reference's correctly rounded divides.
FILE_FLAGS = {"k_mpdata.cu": ["-prec-div=false"], "k_solver.cu": ["-prec-div=false"],
              "k_dynamics.cu": ["-prec-div=false"], "k_subgrid.cu": ["-prec-div=false"]}


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        sorted(glob.glob(os.path.join(HERE, "csrc", "*.h"))) + \
        [os.path.join(ROOT, "include", "dcm.h"), __file__]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(os.path.basename(src), []) + \
            list(extra) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            print(text)
    if failed:
        for src, text in failed:
            sys.stderr.write(f"nvcc failed on {src}:\n{text}\n")
        raise RuntimeError("CUDA build failed")
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
