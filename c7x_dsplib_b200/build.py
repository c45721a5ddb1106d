"""Build the CUDA library libdsplib_b200.so in-tree (sm_100a only).

    python -m c7x_dsplib_b200.build          # incremental
    python -m c7x_dsplib_b200.build --force  # rebuild everything

CUDA sources are compiled by nvcc for ``arch=compute_100a,code=sm_100a`` with
line info; host sources by g++; the CUDA runtime is linked statically so the
library does not depend on whichever libcudart another framework in the
process happens to load.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libdsplib_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", f"-I{INCLUDE}",
              f"-I{CSRC}"] + GENCODE
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA_HOME}/include"]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return max(os.path.getmtime(h) for h in hs) if hs else 0.0


def build(force: bool = False, verbose: bool = False) -> str:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}; set CUDA_HOME")
    os.makedirs(OBJ, exist_ok=True)
    hdr = _headers_mtime()
    objs = []
    changed = force or not os.path.exists(LIB)
    for src in _sources():
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), hdr):
            continue
        changed = True
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
        else:
            cxx = shutil.which("g++") or "g++"
            cmd = [cxx] + CXX_FLAGS + ["-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if changed:
        cmd = [NVCC, "-shared", "-cudart", "static", "-o", LIB] + objs + GENCODE + ["-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
