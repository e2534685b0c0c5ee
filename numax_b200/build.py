"""Build libnmxla.so (sm_100a) in-tree from numax_b200/csrc/*.cu.

The library is compiled by nvcc directly -- no torch extension machinery --
because its interface is a plain C ABI (include/nmx_la.h).  Objects go to
numax_b200/_build/, the shared library to numax_b200/libnmxla.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnmxla.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC,
    # IEEE division and square root, no flush-to-zero: the oracle's rounding.
    "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
]


def cutlass_include() -> str:
    """CUTLASS/CuTe headers (vendored by the flashinfer wheel in this image)."""
    import importlib.util
    spec = importlib.util.find_spec("flashinfer")
    cands = []
    if spec and spec.submodule_search_locations:
        cands.append(os.path.join(spec.submodule_search_locations[0], "data", "cutlass", "include"))
    for c in cands:
        if os.path.exists(os.path.join(c, "cutlass", "cutlass.h")):
            return c
    raise RuntimeError("CUTLASS headers not found (flashinfer/data/cutlass/include)")


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; libnmxla.so cannot be built")
    return path


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + _headers()
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    inc = ["-I", cutlass_include()] if os.path.basename(src) == "gemm_tc.cu" else []
    cmd = [nvcc()] + NVCC_FLAGS + inc + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for o in glob.glob(os.path.join(BUILD, "*.o")):
            os.remove(o)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
