"""Build recipe for libhcblas.so (sm_100a kernels + C++ host library).

    python -m hcblas_b200.build          # incremental
    python -m hcblas_b200.build --clean  # from scratch

CUDA sources (csrc/kernels/*.cu) are compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a -lineinfo); host sources
(csrc/host/*.cpp) by g++; the shared object is linked in-tree as
hcblas_b200/libhcblas.so with the CUDA runtime linked statically, so the
library needs only the NVIDIA driver at run time.  Object files go to
_build/ at the repository root.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libhcblas.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", CXX,
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"] + ARCH
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-Wno-unused-function",
             f"-I{CUDA_HOME}/include"]


def _headers():
    hs = glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
    hs += glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return hs


def _stale(src, obj, newest_header):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def _compile(src, obj, verbose):
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    return src, r.stderr


def build(clean: bool = False, verbose: bool = False, jobs: int = 0) -> str:
    if clean and os.path.isdir(OBJ):
        shutil.rmtree(OBJ)
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "kernels", "*.cu")) +
                  glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    hs = _headers()
    newest = max([os.path.getmtime(h) for h in hs] + [os.path.getmtime(__file__)])
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(s, o, newest):
            todo.append((s, o))
    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            for src, err in ex.map(lambda so: _compile(so[0], so[1], verbose), todo):
                if verbose and err.strip():
                    print(err, file=sys.stderr)
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", CXX, "-o", LIB] + objs + [
            "-cudart", "static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=0)
    args = ap.parse_args()
    print(build(args.clean, args.verbose, args.jobs))
