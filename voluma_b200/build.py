"""Build recipe of the native library: every source compiled for sm_100a by nvcc into
voluma_b200/_lib/libvoluma_b200.so (in-tree, so it travels with the repository snapshot).

    python -m voluma_b200.build        # or __graft_entry__.build()
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libvoluma_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# -fmad=false: no contraction of a*b+c, matching the reference's -ffp-contract=off so row
# updates are bit-identical; the kernels are bandwidth-bound, FMA would buy nothing.
# CUDA sources: nvcc, C++17 (its C++20 front end fails on this toolchain's libstdc++ headers);
# host-only sources (*.cpp: plan, hierarchy, C ABI, serving, level schedules): g++, C++20.
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
                "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I" + os.path.join(ROOT, "include"), "-I" + SRC]
CXX = os.environ.get("CXX_HOST", "g++")
CXXFLAGS = ["-std=c++20", "-O3", "-fPIC", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include"), "-I" + SRC,
            "-I" + os.path.join(CUDA_HOME, "include")]


def sources():
    return sorted(os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    hs = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "voluma_b200.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, hdr_time, verbose):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(src), hdr_time):
        return obj
    if src.endswith(".cpp"):
        # host-only sources: the host compiler, C++20
        cmd = [CXX] + CXXFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-x", "cu", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    ht = _headers_mtime()
    # a change of compiler or flags rebuilds every object
    stamp = os.path.join(OBJ, "flags.txt")
    sig = " ".join([NVCC] + FLAGS + [CXX] + CXXFLAGS)
    if not os.path.exists(stamp) or open(stamp).read() != sig:
        for f in os.listdir(OBJ):
            if f.endswith(".o"):
                os.remove(os.path.join(OBJ, f))
        with open(stamp, "w") as fh:
            fh.write(sig)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, ht, verbose), sources()))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
