"""Build the sm_100a CUDA library libfvg.so in-tree (myfvcomcode_b200/lib/).

--fmad=false keeps every multiply and add separately rounded so the kernels follow the
reference's expression order bit for bit; division and square root stay IEEE-rounded
(the nvcc defaults -prec-div=true -prec-sqrt=true).  The kernel sources that hold FP32
instantiations of the precision form (F32_UNITS) are compiled a second time with
-DFVG_F32_TU and --fmad=true: those kernels are not bit-matched to anything, and
multiply-add contraction only removes roundings from them.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libfvg.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2", "-shared",
]


F32_UNITS = ("k_ext.cu", "k_mom3d.cu", "k_scalar.cu")


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return "g++"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(CSRC, "*.h")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(HERE, "..", "include", "fvg.h"), __file__]
    return any(os.path.getmtime(s) > t for s in deps)


def build(force=False, verbose=False, extra=()):
    """Compile every csrc/*.cu to an object (in parallel, one nvcc per file) and link
    them into libfvg.so."""
    if not force and not needs_build():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    obj_dir = os.path.join(HERE, "lib", "_build")
    os.makedirs(obj_dir, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    objs = []
    units = [(src, os.path.basename(src)[:-3], compile_flags) for src in cu]
    f32_flags = [("--fmad=true" if f == "--fmad=false" else f) for f in compile_flags] + ["-DFVG_F32_TU"]
    units += [(src, os.path.basename(src)[:-3] + "_f32", f32_flags) for src in cu
              if os.path.basename(src) in F32_UNITS]
    for src, name, flags in units:
        obj = os.path.join(obj_dir, name + ".o")
        objs.append(obj)
        cmd = [_nvcc(), "-ccbin", _host_cxx()] + flags + list(extra) + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    errs = []
    for src, pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            errs.append(src + ":\n" + out + err)
        elif verbose and err:
            print(err, file=sys.stderr)
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    cmd = [_nvcc(), "-ccbin", _host_cxx(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
           "-Xcompiler", "-fPIC", "-o", LIB + ".tmp"] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=("-Xptxas", "-v") if "--ptxas" in sys.argv else ())
    print(LIB)
