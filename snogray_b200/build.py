"""Build libsnogray_b200.so in-tree: host C++ with g++ (IEEE float, no FMA
contraction, so bounding boxes and midpoints round like the reference), CUDA
with nvcc for sm_100a only, static CUDA runtime.

    python -m snogray_b200.build [--force]
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libsnogray_b200.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = shutil.which("nvcc") or os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
            "-Wno-unused-function", f"-I{CUDA}/include", f"-I{INCLUDE}"]
# -fmad=false: every float operation rounds on its own, as in the reference's
# parity build (-ffp-contract=off), so the same shading code compiled into two
# kernels (the wave renderer and the streaming engine) gives the same bits.
NVCCFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", *ARCH, "-Xcompiler", "-fPIC",
             "--expt-relaxed-constexpr", f"-I{INCLUDE}", "-Xptxas", "-warn-spills"]


def _sources():
    srcs = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cc", ".cu")):
            srcs.append(os.path.join(CSRC, f))
    return srcs


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "snogray_b200.h"))
    return hs


def _compile(src, force):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, ""
    if src.endswith(".cu"):
        cmd = [NVCC, *NVCCFLAGS, *os.environ.get("SNOG_NVCC_FLAGS", "").split(), "-c", src, "-o", obj]
    else:
        cmd = ["g++", *CXXFLAGS, "-c", src, "-o", obj]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{out.stdout}\n{out.stderr}")
    return obj, out.stderr


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [r[0] for r in results]
    if verbose:
        for _, log in results:
            if log.strip():
                print(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = ["g++", "-shared", "-o", LIB + ".tmp", *objs, f"-L{CUDA}/lib64", "-lcudart_static",
               "-ldl", "-lrt", "-lpthread", "-Wl,--no-undefined"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{out.stdout}\n{out.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
