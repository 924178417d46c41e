"""Compile the CUDA sources into the in-tree shared library ``libflam_b200.so``.

    python -m flam_b200.build          # or: python flam_b200/build.py

nvcc cross-compiles for sm_100a without a GPU.  Each translation unit is
compiled in parallel, then linked with the CUDA runtime (static) into one
C-ABI library whose exports are declared in include/flam.h.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libflam_b200.so")
SOURCES = ["scan.cu", "tree.cu", "compress.cu", "compress_tc.cu", "eliminate.cu", "sweep.cu", "logdet.cu", "diag.cu", "capi.cu", "noalloc.cu", "matvec.cu", "sketch.cu", "predictor.cu", "cpqr_wide.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _compile(src, verbose=False):
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", out]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return out, r.stderr


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "flam.h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(p) <= t for p in deps):
            return LIB
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        res = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if verbose:
        for _, log in res:
            sys.stderr.write(log)
    objs = [o for o, _ in res]
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-Xlinker", "--exclude-libs,ALL",
           "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
