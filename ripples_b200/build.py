"""In-tree build of the ripples_b200 native library (sm_100a only).

Compiles ripples_b200/csrc/*.cu and *.cpp with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links
``ripples_b200/_lib/libripples_b200.so`` plus the drop-in ``imm`` tool.
Objects are rebuilt when a source or any header under csrc/ or include/ is
newer.  Run ``python ripples_b200/build.py`` (not ``-m``: importing the
package loads the library this script builds) or call :func:`build`.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ripples_b200")
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_lib", "obj")
LIB = os.path.join(PKG, "_lib", "libripples_b200.so")
TOOL = os.path.join(PKG, "_lib", "imm_b200")
TOOL_SRC = os.path.join(PKG, "tools", "imm_b200.cpp")
SIM_TOOL = os.path.join(PKG, "_lib", "simulator_b200")
SIM_TOOL_SRC = os.path.join(PKG, "tools", "simulator_b200.cpp")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-O3,-Wall",
    "-I" + INCLUDE, "-I" + CSRC,
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build ripples_b200")
    return cand


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if _stale(obj, [src] + _headers()):
        cmd = [_nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [_nvcc(), "-x", "cu"] + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> str:
    """Builds (incrementally) and returns the path of libripples_b200.so."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-o", LIB] + objs + ["-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # the drop-in imm and simulator command-line tools (host C++ over the C ABI)
    for tool, src in ((TOOL, TOOL_SRC), (SIM_TOOL, SIM_TOOL_SRC)):
        if _stale(tool, [src, LIB] + _headers()):
            cxx = shutil.which("g++") or "g++"
            cmd = [cxx, "-O2", "-std=c++17", "-I" + INCLUDE, src, "-o", tool,
                   "-L" + os.path.dirname(LIB), "-lripples_b200", "-Wl,-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"{os.path.basename(tool)} build failed:\n{r.stdout}\n"
                                   f"{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
