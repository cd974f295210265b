"""Builds graphwalker_b200/lib/libgw_b200.so from csrc/ with nvcc for sm_100a.

The library is built in-tree so that it travels with the source tree; the
CUDA runtime is linked statically, so the only dynamic CUDA dependency is the
driver.  Each translation unit is compiled on its own (in parallel) and
relinked only when a source or header is newer than its object.

    python -m graphwalker_b200.build          # or build() from Python
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libgw_b200.so"
HEADERS = sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "graphwalker_b200.h"])

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    return "nvcc"


def _host_compiler() -> list[str]:
    # the system g++ (an environment CXX wrapper may lack parts of the toolchain)
    return ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    if _stale(obj, [src] + HEADERS):
        cmd = [_nvcc(), *_host_compiler(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles every CUDA source and links the shared library; returns its path."""
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    if ptxas_verbose:
        global NVCC_FLAGS
        NVCC_FLAGS = NVCC_FLAGS + ["-Xptxas", "-v"]
    with cf.ThreadPoolExecutor(max_workers=min(8, len(sources))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), sources))
    if _stale(LIB, objs):
        cmd = [_nvcc(), *_host_compiler(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB),
               *map(str, objs), "-cudart", "static", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv))
