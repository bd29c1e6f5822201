"""In-tree build of libqulacs_b200.so with nvcc for sm_100a.

Every ``csrc/*.cu`` is compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``, every
``csrc/*.cpp`` by nvcc's host compiler, and the objects are linked into
``qulacs_b200/libqulacs_b200.so`` (CUDA runtime linked statically).  Objects go to
``qulacs_b200/_build``.  Rebuilds only what changed.  ``csrc/compat/csim_compat.cpp`` becomes
``qulacs_b200/libcsim_b200.so``: csim's operator names and argument lists over the C ABI.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libqulacs_b200.so")
CSIM_LIB = os.path.join(PKG, "libcsim_b200.so")
CXX = os.environ.get("CXX", "g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", f"-I{ROOT}/include"]
CUFLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj
    cmd = [NVCC, "-c", src, "-o", obj] + CXXFLAGS
    if src.endswith(".cu"):
        cmd += CUFLAGS
    else:
        cmd += ["-x", "c++"] + ARCH
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not (os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs)):
        cmd = [NVCC, "-shared", "-o", LIB] + objs + ARCH + ["-cudart", "static", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_csim_compat(verbose)
    return LIB


def build_csim_compat(verbose: bool = False) -> str:
    """libcsim_b200.so: csim's function names and argument lists (C++ linkage) over libqulacs_b200.so."""
    src = os.path.join(CSRC, "compat", "csim_compat.cpp")
    hdr = os.path.join(ROOT, "include", "qulacs_b200", "csim_compat.hpp")
    if os.path.exists(CSIM_LIB) and os.path.getmtime(CSIM_LIB) >= max(
            os.path.getmtime(src), os.path.getmtime(hdr), os.path.getmtime(LIB)):
        return CSIM_LIB
    cmd = [CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-fvisibility=hidden", f"-I{ROOT}/include", src,
           f"-L{PKG}", "-lqulacs_b200", "-Wl,-rpath,$ORIGIN", "-o", CSIM_LIB]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"libcsim_b200 build failed:\n{r.stdout}\n{r.stderr}")
    return CSIM_LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
